// Kernel chains for the 64^3 grid (FP64 and FP32).
#include "ops_impl.cuh"

const OpsTable *spm_table_64(int prec) {
  return prec == 0 ? spm::Impl<64, double>::table() : spm::Impl<64, float>::table();
}
