/* ugks_oracle_implicit.c -- TEST INFRASTRUCTURE ONLY: ImplicitSteady restatement (filled in below). */
#include "ugks_oracle.h"
int uo_implicit_step(uo_ctx* c, double* out, int nout) { (void)c; (void)out; (void)nout; return -1; }
