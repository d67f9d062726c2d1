// thx_host.h -- host set-up helpers shared by the C ABI translation units.
#pragma once
#include "../../include/theseus_b200.h"

namespace thx {
void lgl_rule(int np, double *x, double *w);
void derivative_operators(int np, const double *x, const double *w, double *D, double *Dhat,
                          double *Dhat2);
bool legendre_vinv(int np, const double *x, double *vinv);
}  // namespace thx
