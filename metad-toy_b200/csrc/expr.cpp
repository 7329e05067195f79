// expr.cpp -- recursive-descent compiler of DIM expressions to stack bytecode.
//
// Grammar (precedence low -> high):
//   expr   := term (('+'|'-') term)*
//   term   := unary (('*'|'/') unary)*
//   unary  := ('-'|'+') unary | power
//   power  := primary ('^' unary)?            (right associative)
//   primary:= number | symbol | pi | e | func '(' expr (',' expr)* ')' | '(' expr ')'
#include "expr.h"

#include <cctype>
#include <cmath>
#include <cstdlib>
#include <cstring>

namespace mtd {

namespace {

struct Func { const char *name; int op; int nargs; };
const Func kFuncs[] = {
    {"sin", EOP_SIN, 1}, {"cos", EOP_COS, 1}, {"tan", EOP_TAN, 1}, {"asin", EOP_ASIN, 1},
    {"acos", EOP_ACOS, 1}, {"atan", EOP_ATAN, 1}, {"exp", EOP_EXP, 1}, {"log", EOP_LOG, 1},
    {"log10", EOP_LOG10, 1}, {"sqrt", EOP_SQRT, 1}, {"abs", EOP_ABS, 1}, {"tanh", EOP_TANH, 1},
    {"sinh", EOP_SINH, 1}, {"cosh", EOP_COSH, 1}, {"min", EOP_MIN, 2}, {"max", EOP_MAX, 2},
    {"pow", EOP_POW, 2}, {"atan2", EOP_ATAN2, 2},
};

struct Parser {
    const std::string &s;
    const std::vector<std::string> &syms;
    std::vector<ExprInstr> &code;
    size_t p = 0;
    std::string err;

    void ws() { while (p < s.size() && std::isspace((unsigned char)s[p])) ++p; }
    bool fail(const std::string &m) { if (err.empty()) err = m; return false; }
    void emit(int op, int arg = 0, double val = 0.0) { code.push_back(ExprInstr{op, arg, val}); }

    bool expr() {
        if (!term()) return false;
        for (;;) {
            ws();
            if (p < s.size() && (s[p] == '+' || s[p] == '-')) {
                char o = s[p++];
                if (!term()) return false;
                emit(o == '+' ? EOP_ADD : EOP_SUB);
            } else return true;
        }
    }
    bool term() {
        if (!unary()) return false;
        for (;;) {
            ws();
            if (p < s.size() && (s[p] == '*' || s[p] == '/')) {
                char o = s[p++];
                if (!unary()) return false;
                emit(o == '*' ? EOP_MUL : EOP_DIV);
            } else return true;
        }
    }
    bool unary() {
        ws();
        if (p < s.size() && s[p] == '-') { ++p; if (!unary()) return false; emit(EOP_NEG); return true; }
        if (p < s.size() && s[p] == '+') { ++p; return unary(); }
        return power();
    }
    bool power() {
        if (!primary()) return false;
        ws();
        if (p < s.size() && s[p] == '^') {
            ++p;
            if (!unary()) return false;
            emit(EOP_POW);
        }
        return true;
    }
    bool primary() {
        ws();
        if (p >= s.size()) return fail("unexpected end of expression");
        char ch = s[p];
        if (std::isdigit((unsigned char)ch) || ch == '.') {
            const char *b = s.c_str() + p;
            char *e = nullptr;
            double v = std::strtod(b, &e);
            if (e == b) return fail("bad number");
            p += (size_t)(e - b);
            emit(EOP_CONST, 0, v);
            return true;
        }
        if (std::isalpha((unsigned char)ch) || ch == '_') {
            size_t q = p;
            while (q < s.size() && (std::isalnum((unsigned char)s[q]) || s[q] == '_')) ++q;
            std::string id = s.substr(p, q - p);
            p = q;
            ws();
            if (p < s.size() && s[p] == '(') {
                ++p;
                const Func *f = nullptr;
                for (const Func &k : kFuncs)
                    if (id == k.name) f = &k;
                if (!f) return fail("unknown function '" + id + "'");
                for (int a = 0; a < f->nargs; ++a) {
                    if (a > 0) {
                        ws();
                        if (p >= s.size() || s[p] != ',') return fail("expected ',' in call of " + id);
                        ++p;
                    }
                    if (!expr()) return false;
                }
                ws();
                if (p >= s.size() || s[p] != ')') return fail("expected ')' after arguments of " + id);
                ++p;
                emit(f->op);
                return true;
            }
            for (size_t k = 0; k < syms.size(); ++k)
                if (syms[k] == id) { emit(EOP_SYM, (int)k); return true; }
            if (id == "pi") { emit(EOP_CONST, 0, 3.14159265358979323846); return true; }
            if (id == "e") { emit(EOP_CONST, 0, 2.71828182845904523536); return true; }
            return fail("unknown symbol '" + id + "'");
        }
        if (ch == '(') {
            ++p;
            if (!expr()) return false;
            ws();
            if (p >= s.size() || s[p] != ')') return fail("expected ')'");
            ++p;
            return true;
        }
        return fail(std::string("unexpected character '") + ch + "'");
    }
};

}  // namespace

std::string compile_expr(const std::string &src, const std::vector<std::string> &symbols, std::vector<ExprInstr> &code) {
    code.clear();
    Parser ps{src, symbols, code};
    if (!ps.expr()) return "ExprTk Error: " + ps.err + " in \"" + src + "\"";
    ps.ws();
    if (ps.p != src.size()) return "ExprTk Error: trailing characters in \"" + src + "\"";
    if ((int)code.size() > kMaxExprLen) return "Error: DIM expression too long: \"" + src + "\"";
    int depth = 0, maxd = 0;
    for (auto &c : code) {
        if (c.op == EOP_CONST || c.op == EOP_SYM) depth++;
        else if (c.op == EOP_ADD || c.op == EOP_SUB || c.op == EOP_MUL || c.op == EOP_DIV || c.op == EOP_POW ||
                 c.op == EOP_MIN || c.op == EOP_MAX || c.op == EOP_ATAN2) depth--;
        if (depth > maxd) maxd = depth;
    }
    if (maxd > kMaxExprStack) return "Error: DIM expression nests too deeply: \"" + src + "\"";
    return "";
}

double eval_expr_host(const std::vector<ExprInstr> &code, const double *sym, int nsym, double *grad) {
    struct D { double v; double g[16]; };
    D st[kMaxExprStack];
    int sp = 0;
    auto un = [&](D &a, double v, double dv) { for (int k = 0; k < nsym; ++k) a.g[k] *= dv; a.v = v; };
    for (const ExprInstr &c : code) {
        switch (c.op) {
        case EOP_CONST: st[sp].v = c.val; for (int k = 0; k < nsym; ++k) st[sp].g[k] = 0; ++sp; break;
        case EOP_SYM: st[sp].v = sym[c.arg]; for (int k = 0; k < nsym; ++k) st[sp].g[k] = (k == c.arg); ++sp; break;
        case EOP_NEG: un(st[sp - 1], -st[sp - 1].v, -1.0); break;
        case EOP_ADD: case EOP_SUB: case EOP_MUL: case EOP_DIV: case EOP_POW:
        case EOP_MIN: case EOP_MAX: case EOP_ATAN2: {
            D &a = st[sp - 2], &b = st[sp - 1];
            double v, da, db;
            switch (c.op) {
            case EOP_ADD: v = a.v + b.v; da = 1; db = 1; break;
            case EOP_SUB: v = a.v - b.v; da = 1; db = -1; break;
            case EOP_MUL: v = a.v * b.v; da = b.v; db = a.v; break;
            case EOP_DIV: v = a.v / b.v; da = 1.0 / b.v; db = -a.v / (b.v * b.v); break;
            case EOP_POW: v = std::pow(a.v, b.v); da = b.v * std::pow(a.v, b.v - 1.0); db = (a.v > 0) ? v * std::log(a.v) : 0.0; break;
            case EOP_MIN: v = a.v <= b.v ? a.v : b.v; da = a.v <= b.v; db = !(a.v <= b.v); break;
            case EOP_MAX: v = a.v >= b.v ? a.v : b.v; da = a.v >= b.v; db = !(a.v >= b.v); break;
            default: { double r2 = a.v * a.v + b.v * b.v; v = std::atan2(a.v, b.v); da = b.v / r2; db = -a.v / r2; }
            }
            for (int k = 0; k < nsym; ++k) a.g[k] = da * a.g[k] + db * b.g[k];
            a.v = v;
            --sp;
            break;
        }
        default: {
            D &a = st[sp - 1];
            double x = a.v, v = 0, dv = 0;
            switch (c.op) {
            case EOP_SIN: v = std::sin(x); dv = std::cos(x); break;
            case EOP_COS: v = std::cos(x); dv = -std::sin(x); break;
            case EOP_TAN: v = std::tan(x); dv = 1.0 + v * v; break;
            case EOP_ASIN: v = std::asin(x); dv = 1.0 / std::sqrt(1.0 - x * x); break;
            case EOP_ACOS: v = std::acos(x); dv = -1.0 / std::sqrt(1.0 - x * x); break;
            case EOP_ATAN: v = std::atan(x); dv = 1.0 / (1.0 + x * x); break;
            case EOP_EXP: v = std::exp(x); dv = v; break;
            case EOP_LOG: v = std::log(x); dv = 1.0 / x; break;
            case EOP_LOG10: v = std::log10(x); dv = 1.0 / (x * 2.30258509299404568402); break;
            case EOP_SQRT: v = std::sqrt(x); dv = 0.5 / v; break;
            case EOP_ABS: v = std::fabs(x); dv = (x > 0) - (x < 0); break;
            case EOP_TANH: v = std::tanh(x); dv = 1.0 - v * v; break;
            case EOP_SINH: v = std::sinh(x); dv = std::cosh(x); break;
            case EOP_COSH: v = std::cosh(x); dv = std::sinh(x); break;
            }
            un(a, v, dv);
        }
        }
    }
    if (grad)
        for (int k = 0; k < nsym; ++k) grad[k] = st[0].g[k];
    return st[0].v;
}

}  // namespace mtd
