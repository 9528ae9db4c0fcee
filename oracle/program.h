// Program descriptor shared by the oracle and its tests (TEST INFRASTRUCTURE).
//
// The descriptor is this repository's flat encoding of a compiled loom
// board.Program restricted to what the Poseidon2 prove path consumes
// (board/program.go:21-89): modules with their sizes and relations, the
// columns they reference, grand-product prover steps, and the per-round
// staged (committed) columns after board.Compile's sweep
// (board/rounds.go:219-292).  Layout, little-endian u32 words:
//
//   magic 0x3150474C, n_rounds, n_modules, n_columns, n_nodes, n_steps
//   module  : log_n, str name, n_rel, rel_root[n_rel]
//   column  : str name, module, field(0 base|1 ext), kind(0 witness|1 step
//             output|2 Lagrange verifier column), param(int32 row; <0 means
//             relative from the end, -(i+1))
//   node    : op(0 col|1 coin|2 const|3 add|4 sub|5 mul), a, b
//             col: a = column, b = shift (int32); coin: a = round;
//             const: a = canonical value; add/sub/mul: a, b = child nodes
//             (children precede parents)
//   step    : type(0 grand product), round, module, num_node, den_node, out_col
//   round   : n_staged, col[n_staged]
//   str     : byte length, then the bytes packed 4 per word
#pragma once
#include <cstdint>
#include <string>
#include <vector>

namespace orc {

enum { OP_COL = 0, OP_COIN = 1, OP_CONST = 2, OP_ADD = 3, OP_SUB = 4, OP_MUL = 5 };
enum { KIND_WITNESS = 0, KIND_STEP = 1, KIND_LAGRANGE = 2 };

struct PModule { uint32_t log_n; std::string name; std::vector<uint32_t> rels; };
struct PColumn { std::string name; uint32_t module, field, kind; int32_t param; };
struct PNode { uint32_t op, a, b; };
struct PStep { uint32_t type, round, module, num, den, out; };
struct Program {
  uint32_t n_rounds = 0;
  std::vector<PModule> modules;
  std::vector<PColumn> columns;
  std::vector<PNode> nodes;
  std::vector<PStep> steps;
  std::vector<std::vector<uint32_t>> staged;
};
Program parse_program(const uint32_t* w, size_t n);

}  // namespace orc
