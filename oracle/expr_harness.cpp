// expr_harness.cpp -- TEST INFRASTRUCTURE ONLY.
//
// Compiles DIM expressions with exprtk (third_party/exprtk.hpp of the
// reference checkout, the library src/grids/DimSet.cu:54-97 uses) and
// evaluates them the way the reference does: a symbol table with one variable
// per symbol and no add_constants() (src/grids/DimSet.cu:11-16, :46-50),
// parser<double> with default settings, value() for the DIM value and
// exprtk::derivative(expression, name) for dS/dv.  The header is read from the
// reference checkout at build time (oracle/Makefile, target `ref`); nothing of
// it is copied here.  Used only to generate golden vectors for the tests of
// the expression compiler.
#include <cstring>
#include <string>
#include <vector>

#include "exprtk.hpp"

extern "C" {

// Returns 0 and fills value and grad[nsym] on success; 1 with the parser's
// message in err on a compile error.
int exref_eval(const char *expr, int nsym, const char *const *names, const double *values, double *value,
               double *grad, char *err, int errlen) {
    std::vector<double> var(values, values + nsym);
    exprtk::symbol_table<double> st;
    for (int k = 0; k < nsym; ++k) st.add_variable(names[k], var[k]);
    exprtk::expression<double> e;
    e.register_symbol_table(st);
    exprtk::parser<double> parser;
    if (!parser.compile(expr, e)) {
        if (err && errlen > 0) {
            std::strncpy(err, parser.error().c_str(), (size_t)errlen - 1);
            err[errlen - 1] = '\0';
        }
        return 1;
    }
    *value = e.value();
    for (int k = 0; k < nsym; ++k) grad[k] = exprtk::derivative(e, std::string(names[k]));
    return 0;
}

}  // extern "C"
