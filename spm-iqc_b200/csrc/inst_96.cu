// Kernel chains for the 96^3 grid (FP64 and FP32).
#include "ops_impl.cuh"

const OpsTable *spm_table_96(int prec) {
  return prec == 0 ? spm::Impl<96, double>::table() : spm::Impl<96, float>::table();
}
