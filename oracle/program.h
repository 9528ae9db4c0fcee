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
//             output|2 Lagrange verifier column|3 setup column), param(int32
//             row; <0 means relative from the end, -(i+1))
//   node    : op(0 col|1 coin|2 const|3 add|4 sub|5 mul|6 exposed average),
//             a, b.  col: a = column, b = shift (int32); coin: a = round;
//             const: a = canonical value; add/sub/mul: a, b = child nodes
//             (children precede parents); exposed average: a = exposed value
//             (the a-th exposing step's value), value total / N of the
//             module evaluating it (expr/ast.go:223-227); 7 exposed value:
//             a = exposed value index, the value itself (a constant)
//   step    : type 0 grand product: 0, round, module, num_node, den_node, out_col
//             type 1 lookup multiplicities (width-1 tables): 1, round, n_src,
//               n_tgt, src_node[n_src], tgt_node[n_tgt], out_col[n_tgt]
//             type 2 cyclic logup: 2, round, module, out_col, n_terms,
//               (E_node, M_node)[n_terms]; its total is exposed
//             type 3 running ratio: 3, round, module, num_node, den_node,
//               out_col; its end is exposed (board/product.go:72-198)
//             type 4 lookup multiplicities of tuples with optional selectors:
//               4, round, width, n_src, n_tgt, flags (bit 0: source
//               selectors, bit 1: target selectors), src_sel[n_src],
//               tgt_sel[n_tgt] (when flagged), src nodes [n_src x width],
//               tgt nodes [n_tgt x width], out_col[n_tgt]
//             Exposed values are numbered in step order over types 2 and 3.
//   round   : n_staged, col[n_staged]
//   str     : byte length, then the bytes packed 4 per word
#pragma once
#include <cstdint>
#include <string>
#include <vector>

namespace orc {

enum { OP_COL = 0, OP_COIN = 1, OP_CONST = 2, OP_ADD = 3, OP_SUB = 4, OP_MUL = 5, OP_EXPAVG = 6, OP_EXPVAL = 7 };
enum { STEP_GP = 0, STEP_MULT = 1, STEP_LOGUP = 2, STEP_RATIO = 3, STEP_MULTW = 4 };
enum { KIND_WITNESS = 0, KIND_STEP = 1, KIND_LAGRANGE = 2, KIND_SETUP = 3 };

struct PModule { uint32_t log_n; std::string name; std::vector<uint32_t> rels; };
struct PColumn { std::string name; uint32_t module, field, kind; int32_t param; };
struct PNode { uint32_t op, a, b; };
struct PStep {
  uint32_t type, round, module = 0, num = 0, den = 0, out = 0;
  std::vector<uint32_t> src, tgt, outs;   // multiplicities (type 4: width nodes per table, table-major)
  uint32_t width = 1, flags = 0;          // type 4: tuple width; bit 0 source selectors, bit 1 target selectors
  std::vector<uint32_t> sel_s, sel_t;     // type 4 selectors
  std::vector<uint32_t> e, m;             // logup terms M/E
  uint32_t exposed = 0;                   // logup: index of its exposed total
};
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
