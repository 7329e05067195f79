// expr.h -- DIM expressions compiled to a small stack bytecode that the bias
// kernel evaluates on the device with forward-mode derivatives.
//
// It replaces the exprtk expressions and exprtk::derivative of
// src/grids/DimSet.cu:54-97: the value is the same expression, and the chain
// factor dS/dv is exact instead of exprtk's five-point difference (h = 1e-8,
// which adds ~1e-8 relative noise to the reference's forces).  The grammar is
// exprtk's expression subset (no statements, assignments, strings, vectors or
// loops); the operations and their semantics are listed in expr_ops.h.
#pragma once

#include <string>
#include <vector>

#include "expr_ops.h"

namespace mtd {

struct ExprInstr {
    int op;
    int arg;      // symbol index for EOP_SYM
    double val;   // constant for EOP_CONST
};

constexpr int kMaxExprLen = 64;
constexpr int kMaxExprStack = 16;

// Compiles `src` over the symbol names; returns "" on success or an error message.
std::string compile_expr(const std::string &src, const std::vector<std::string> &symbols, std::vector<ExprInstr> &code);

// Host evaluation of the same bytecode (value and d/dsym), used by the parser's
// own validation and by tests of the compiler.
double eval_expr_host(const std::vector<ExprInstr> &code, const double *sym, int nsym, double *grad);

}  // namespace mtd
