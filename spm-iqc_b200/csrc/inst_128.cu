// Kernel chains for the 128^3 grid (FP64 and FP32).
#include "ops_impl.cuh"

const OpsTable *spm_table_128(int prec) {
  return prec == 0 ? spm::Impl<128, double>::table() : spm::Impl<128, float>::table();
}
