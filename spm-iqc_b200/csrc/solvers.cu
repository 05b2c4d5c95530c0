// Host-side solvers built on the transform kernels (filled in below).
#include "spm_internal.h"

void spm_free_extra(spm_ctx *c) { (void)c; }
