// Kernel chains for the 192^3 grid (FP64 and FP32).
#include "ops_impl.cuh"

const OpsTable *spm_table_192(int prec) {
  return prec == 0 ? spm::Impl<192, double>::table() : spm::Impl<192, float>::table();
}
