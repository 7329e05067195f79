// expr.cpp -- compiler of DIM expressions to stack bytecode.
//
// The expression language is the one exprtk::parser<double> accepts with its
// default settings for a single expression (src/grids/DimSet.cu:54-66):
//
//   precedence (low -> high), left-associative unless noted
//     c ? a : b                       (whole expression as condition; right-assoc.)
//     or | nor xor xnor
//     and & nand
//     < <= > >= == = != <>
//     + -
//     * / %
//     unary -  (binds looser than ^:  -a^b = -(a^b))
//     ^                                (right-assoc.)
//   primaries: numbers, symbols, true/false, pi/e, ( ) [ ] { } groups,
//     func(args): the functions of expr_ops.h, if(c, a, b), and the variadic
//     min max sum avg mul mand mor.
//   Names of functions, keywords and symbols match case-insensitively.
//   Implicit multiplication as exprtk inserts it: number then symbol or
//   bracket ("2v1", "2(v1+1)"), symbol then number or symbol ("v1 v2"), a
//   variable then a bracket ("v1(v2)"), and a closing bracket then number or
//   symbol ("(v1+1)v2").
//
// Deviations: `pi` and `e` are accepted as constants (exprtk needs
// add_constants() for them, which the reference leaves out, so it rejects
// them; a symbol of that name wins).  Assignment (":=", which exprtk accepts
// and which would overwrite a CV), statements, strings, vectors, loops and
// switch are not expressions of a DIM and give a parse error.
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
    {"sinh", EOP_SINH, 1}, {"cosh", EOP_COSH, 1}, {"not", EOP_NOT, 1}, {"sgn", EOP_SGN, 1},
    {"floor", EOP_FLOOR, 1}, {"ceil", EOP_CEIL, 1}, {"round", EOP_ROUND, 1}, {"trunc", EOP_TRUNC, 1},
    {"frac", EOP_FRAC, 1}, {"sec", EOP_SEC, 1}, {"csc", EOP_CSC, 1}, {"cot", EOP_COT, 1},
    {"asinh", EOP_ASINH, 1}, {"acosh", EOP_ACOSH, 1}, {"atanh", EOP_ATANH, 1}, {"log2", EOP_LOG2, 1},
    {"log1p", EOP_LOG1P, 1}, {"expm1", EOP_EXPM1, 1}, {"erf", EOP_ERF, 1}, {"erfc", EOP_ERFC, 1},
    {"ncdf", EOP_NCDF, 1}, {"sinc", EOP_SINC, 1}, {"deg2rad", EOP_DEG2RAD, 1}, {"rad2deg", EOP_RAD2DEG, 1},
    {"deg2grad", EOP_DEG2GRAD, 1}, {"grad2deg", EOP_GRAD2DEG, 1},
    {"pow", EOP_POW, 2}, {"atan2", EOP_ATAN2, 2}, {"mod", EOP_MOD, 2}, {"hypot", EOP_HYPOT, 2},
    {"logn", EOP_LOGN, 2}, {"root", EOP_ROOT, 2}, {"roundn", EOP_ROUNDN, 2}, {"equal", EOP_EQUAL, 2},
    {"not_equal", EOP_NEQUAL, 2}, {"shl", EOP_SHL, 2}, {"shr", EOP_SHR, 2},
    {"if", EOP_SEL, 3}, {"clamp", EOP_CLAMP, 3}, {"iclamp", EOP_ICLAMP, 3}, {"inrange", EOP_INRANGE, 3},
};

// Variadic functions: folded left to right over binary operations.
struct VarFunc { const char *name; int op; };
const VarFunc kVarFuncs[] = {
    {"min", EOP_MIN}, {"max", EOP_MAX}, {"sum", EOP_ADD}, {"avg", EOP_ADD}, {"mul", EOP_MUL},
    {"mand", EOP_AND}, {"mor", EOP_OR},
};

// exprtk's reserved words: no implicit multiplication next to them.
const char *const kReserved[] = {
    "assert", "break", "case", "continue", "const", "default", "false", "for", "if", "else", "ilike", "in",
    "like", "and", "nand", "nor", "not", "null", "or", "repeat", "return", "shl", "shr", "swap", "switch",
    "true", "until", "var", "while", "xnor", "xor",
};

std::string lower(const std::string &s) {
    std::string r(s);
    for (char &c : r) c = (char)std::tolower((unsigned char)c);
    return r;
}

bool reserved(const std::string &id) {
    const std::string l = lower(id);
    for (const char *w : kReserved)
        if (l == w) return true;
    return false;
}

enum TokKind { T_NUM, T_ID, T_OP, T_END };

struct Tok {
    TokKind kind;
    std::string text;   // identifier or operator
    double val = 0.0;
};

bool is_open(const Tok &t) { return t.kind == T_OP && (t.text == "(" || t.text == "[" || t.text == "{"); }
bool is_close(const Tok &t) { return t.kind == T_OP && (t.text == ")" || t.text == "]" || t.text == "}"); }
bool plain_id(const Tok &t) { return t.kind == T_ID && !reserved(t.text); }
bool is_function(const std::string &id);

std::string lex(const std::string &s, std::vector<Tok> &out) {
    size_t p = 0;
    while (p < s.size()) {
        const char ch = s[p];
        if (std::isspace((unsigned char)ch)) { ++p; continue; }
        if (std::isdigit((unsigned char)ch) || (ch == '.' && p + 1 < s.size() && std::isdigit((unsigned char)s[p + 1]))) {
            size_t q = p;
            while (q < s.size() && std::isdigit((unsigned char)s[q])) ++q;
            if (q < s.size() && s[q] == '.') {
                ++q;
                while (q < s.size() && std::isdigit((unsigned char)s[q])) ++q;
            }
            if (q < s.size() && (s[q] == 'e' || s[q] == 'E')) {
                size_t r = q + 1;
                if (r < s.size() && (s[r] == '+' || s[r] == '-')) ++r;
                if (r < s.size() && std::isdigit((unsigned char)s[r])) {
                    while (r < s.size() && std::isdigit((unsigned char)s[r])) ++r;
                    q = r;
                }
            }
            Tok t{T_NUM, s.substr(p, q - p)};
            t.val = std::strtod(t.text.c_str(), nullptr);
            out.push_back(t);
            p = q;
            continue;
        }
        if (std::isalpha((unsigned char)ch) || ch == '_') {
            size_t q = p + 1;
            while (q < s.size() && (std::isalnum((unsigned char)s[q]) || s[q] == '_' || s[q] == '.')) ++q;
            out.push_back(Tok{T_ID, s.substr(p, q - p)});
            p = q;
            continue;
        }
        if (ch == '&' || ch == '|') {
            out.push_back(Tok{T_ID, ch == '&' ? "and" : "or"});
            ++p;
            continue;
        }
        static const char *const two[] = {"<=", ">=", "==", "!=", "<>", ":="};
        bool matched = false;
        for (const char *t : two)
            if (s.compare(p, 2, t) == 0) {
                if (t[0] == ':') return "assignment is not an expression";
                out.push_back(Tok{T_OP, t});
                p += 2;
                matched = true;
                break;
            }
        if (matched) continue;
        if (std::strchr("+-*/%^<>=()[]{},?:", ch)) {
            out.push_back(Tok{T_OP, std::string(1, ch)});
            ++p;
            continue;
        }
        return std::string("unexpected character '") + ch + "'";
    }
    // implicit multiplication
    std::vector<Tok> r;
    for (size_t i = 0; i < out.size(); ++i) {
        if (i > 0) {
            const Tok &a = out[i - 1], &b = out[i];
            const bool ins = (a.kind == T_NUM && (plain_id(b) || is_open(b))) ||
                             (plain_id(a) && (b.kind == T_NUM || plain_id(b))) ||
                             (plain_id(a) && is_open(b) && !is_function(a.text)) ||   // "v1(v2)"
                             (is_close(a) && (b.kind == T_NUM || plain_id(b)));
            if (ins) r.push_back(Tok{T_OP, "*"});
        }
        r.push_back(out[i]);
    }
    r.push_back(Tok{T_END, ""});
    out.swap(r);
    return "";
}

bool is_function(const std::string &id) {
    const std::string l = lower(id);
    for (const Func &f : kFuncs)
        if (l == f.name) return true;
    for (const VarFunc &f : kVarFuncs)
        if (l == f.name) return true;
    return false;
}

struct BinOp { int left, right, op; };

// Binary operator at token t (false if t is none).
bool binop(const Tok &t, BinOp &b) {
    if (t.kind == T_OP) {
        const std::string &o = t.text;
        if (o == "+") b = {7, 8, EOP_ADD};
        else if (o == "-") b = {7, 8, EOP_SUB};
        else if (o == "*") b = {10, 11, EOP_MUL};
        else if (o == "/") b = {10, 11, EOP_DIV};
        else if (o == "%") b = {10, 11, EOP_MOD};
        else if (o == "^") b = {12, 12, EOP_POW};
        else if (o == "<") b = {5, 6, EOP_LT};
        else if (o == "<=") b = {5, 6, EOP_LE};
        else if (o == ">") b = {5, 6, EOP_GT};
        else if (o == ">=") b = {5, 6, EOP_GE};
        else if (o == "==" || o == "=") b = {5, 6, EOP_EQ};
        else if (o == "!=" || o == "<>") b = {5, 6, EOP_NE};
        else return false;
        return true;
    }
    if (t.kind == T_ID) {
        const std::string o = lower(t.text);
        if (o == "and") b = {3, 4, EOP_AND};
        else if (o == "nand") b = {3, 4, EOP_NAND};
        else if (o == "or") b = {1, 2, EOP_OR};
        else if (o == "nor") b = {1, 2, EOP_NOR};
        else if (o == "xor") b = {1, 2, EOP_XOR};
        else if (o == "xnor") b = {1, 2, EOP_XNOR};
        else return false;
        return true;
    }
    return false;
}

struct Parser {
    const std::vector<Tok> &t;
    const std::vector<std::string> &syms;
    std::vector<ExprInstr> &code;
    size_t p = 0;
    int depth = 0;
    std::string err;

    const Tok &cur() const { return t[p]; }
    bool op_is(const char *s) const { return cur().kind == T_OP && cur().text == s; }
    bool fail(const std::string &m) { if (err.empty()) err = m; return false; }
    void emit(int op, int arg = 0, double val = 0.0) { code.push_back(ExprInstr{op, arg, val}); }

    bool expression(int prec) {
        if (++depth > 64) return fail("expression nests too deeply");
        if (!branch(prec)) return false;
        for (;;) {
            BinOp b;
            if (!binop(cur(), b) || b.left < prec) break;
            ++p;
            if (!expression(b.right)) return false;
            emit(b.op);
        }
        if (prec == 0 && op_is("?")) {   // the whole expression is the condition
            ++p;
            if (!expression(0)) return false;
            if (!op_is(":")) return fail("expected ':' in a conditional");
            ++p;
            if (!expression(0)) return false;
            emit(EOP_SEL);
        }
        --depth;
        return true;
    }

    bool close(const std::string &open) {
        const char *want = open == "(" ? ")" : (open == "[" ? "]" : "}");
        if (!op_is(want)) return fail(std::string("expected '") + want + "'");
        ++p;
        return true;
    }

    // Arguments of a call: ( expr (, expr)* ); returns the count.
    bool args(const std::string &name, int &n) {
        const std::string open = cur().text;
        ++p;
        n = 0;
        if (is_close(cur())) return fail("call of " + name + " without arguments");
        for (;;) {
            if (!expression(0)) return false;
            ++n;
            if (op_is(",")) { ++p; continue; }
            return close(open);
        }
    }

    bool branch(int prec) {
        (void)prec;
        const Tok &k = cur();
        if (k.kind == T_OP && k.text == "-") {
            ++p;
            if (!expression(11)) return false;
            emit(EOP_NEG);
            return true;
        }
        if (k.kind == T_OP && k.text == "+") {
            ++p;
            return expression(13);
        }
        if (k.kind == T_NUM) {
            emit(EOP_CONST, 0, k.val);
            ++p;
            return true;
        }
        if (is_open(k)) {
            const std::string open = k.text;
            ++p;
            if (!expression(0)) return false;
            return close(open);
        }
        if (k.kind == T_ID) {
            const std::string id = k.text, l = lower(k.text);
            ++p;
            if (is_open(cur())) {
                for (const Func &f : kFuncs)
                    if (l == f.name) {
                        int n = 0;
                        if (!args(id, n)) return false;
                        if (n != f.nargs)
                            return fail(id + " takes " + std::to_string(f.nargs) + " argument(s), got " +
                                        std::to_string(n));
                        emit(f.op);
                        return true;
                    }
                for (const VarFunc &f : kVarFuncs)
                    if (l == f.name) {
                        int n = 0;
                        if (!args(id, n)) return false;
                        return fold(l, f.op, n);
                    }
            }
            for (size_t s = 0; s < syms.size(); ++s)
                if (syms[s] == id) { emit(EOP_SYM, (int)s); return true; }
            for (size_t s = 0; s < syms.size(); ++s)
                if (lower(syms[s]) == l) { emit(EOP_SYM, (int)s); return true; }
            if (l == "true") { emit(EOP_CONST, 0, 1.0); return true; }
            if (l == "false") { emit(EOP_CONST, 0, 0.0); return true; }
            if (l == "pi") { emit(EOP_CONST, 0, 3.14159265358979323846); return true; }
            if (l == "e") { emit(EOP_CONST, 0, 2.71828182845904523536); return true; }
            if (is_open(cur())) return fail("unknown function '" + id + "'");
            return fail("unknown symbol '" + id + "'");
        }
        if (k.kind == T_END) return fail("unexpected end of expression");
        return fail("unexpected '" + k.text + "'");
    }

    // A left fold ((a0 op a1) op a2) ... of the n arguments just compiled.
    // Their code is n contiguous blocks that each leave one value; it is
    // re-emitted as a0 a1 op a2 op ... so the stack holds at most two of them.
    bool fold(const std::string &name, int op, int n) {
        if (n == 1) {
            if (op == EOP_AND || op == EOP_OR) {   // truth value of the one argument
                emit(EOP_CONST, 0, 0.0);
                emit(EOP_NE);
            }
            return true;
        }
        // split the trailing code into the n argument blocks by stack effect
        std::vector<size_t> start(n);
        size_t pos = code.size();
        for (int a = n - 1; a >= 0; --a) {
            int need = 1;   // values this block must leave
            while (need > 0) {
                --pos;
                need += expr_arity(code[pos].op) - 1;
            }
            start[a] = pos;
        }
        std::vector<ExprInstr> tail(code.begin() + (long)start[0], code.end());
        code.resize(start[0]);
        for (int a = 0; a < n; ++a) {
            const size_t b = start[a] - start[0];
            const size_t e = (a + 1 < n ? start[a + 1] : start[0] + tail.size()) - start[0];
            code.insert(code.end(), tail.begin() + (long)b, tail.begin() + (long)e);
            if (a > 0) emit(op);
        }
        if (name == "avg") {
            emit(EOP_CONST, 0, (double)n);
            emit(EOP_DIV);
        }
        return true;
    }
};

}  // namespace

std::string compile_expr(const std::string &src, const std::vector<std::string> &symbols, std::vector<ExprInstr> &code) {
    code.clear();
    std::vector<Tok> toks;
    std::string e = lex(src, toks);
    if (!e.empty()) return "ExprTk Error: " + e + " in \"" + src + "\"";
    Parser ps{toks, symbols, code};
    if (!ps.expression(0)) return "ExprTk Error: " + ps.err + " in \"" + src + "\"";
    if (ps.cur().kind != T_END) return "ExprTk Error: unexpected '" + ps.cur().text + "' in \"" + src + "\"";
    if ((int)code.size() > kMaxExprLen) return "Error: DIM expression too long: \"" + src + "\"";
    int depth = 0, maxd = 0;
    for (auto &c : code) {
        depth += 1 - expr_arity(c.op);
        if (depth > maxd) maxd = depth;
    }
    if (maxd > kMaxExprStack) return "Error: DIM expression nests too deeply: \"" + src + "\"";
    return "";
}

double eval_expr_host(const std::vector<ExprInstr> &code, const double *sym, int nsym, double *grad) {
    struct D { double v; double g[16]; };
    D st[kMaxExprStack];
    int sp = 0;
    for (const ExprInstr &c : code) {
        if (c.op == EOP_CONST || c.op == EOP_SYM) {
            st[sp].v = c.op == EOP_CONST ? c.val : sym[c.arg];
            for (int k = 0; k < nsym; ++k) st[sp].g[k] = (c.op == EOP_SYM && k == c.arg) ? 1.0 : 0.0;
            ++sp;
            continue;
        }
        const int n = expr_arity(c.op);
        double a[3] = {0, 0, 0}, d[3];
        for (int i = 0; i < n; ++i) a[i] = st[sp - n + i].v;
        const double v = expr_apply(c.op, a, d);
        D &r = st[sp - n];
        for (int k = 0; k < nsym; ++k) {
            double g = 0.0;
            for (int i = 0; i < n; ++i)
                if (d[i] != 0.0) g += d[i] * st[sp - n + i].g[k];
            r.g[k] = g;
        }
        r.v = v;
        sp -= n - 1;
    }
    if (grad)
        for (int k = 0; k < nsym; ++k) grad[k] = st[0].g[k];
    return st[0].v;
}

}  // namespace mtd
