// Per-(grid size, precision) entry points into the kernel chains. Each
// inst_<N>.cu translation unit provides the tables of one grid size, so the
// sizes compile in parallel.
#pragma once

struct spm_ctx;

struct OpsTable {
  int (*fft)(spm_ctx *, const void *x, void *xhat);
  int (*ifft)(spm_ctx *, const void *xhat, void *x);
  int (*energy)(spm_ctx *, const void *phi, const void *uhat);
  int (*grad_step)(spm_ctx *, void *phi, void *uhat);
  int (*grad_steps)(spm_ctx *, void *phi, void *uhat, int nsteps);
  int (*grad_steps_ev)(spm_ctx *, void *phi, void *uhat, int nsteps, void *const *events);
  int (*grad_step_ev)(spm_ctx *, void *phi, void *uhat, void *const *events);
  int (*ngrad)(spm_ctx *, const void *phi, void *grad);
  int (*hv)(spm_ctx *, const void *phi, const void *const *v, void *const *hv, int n);
  int (*precond)(spm_ctx *, void *const *w, int n);
  int (*dot)(spm_ctx *, const void *p, const void *q);
  int (*tangent)(spm_ctx *, const void *phi0, const void *phi1, void *v_out, void *vhat, void *gv);
  int (*force)(spm_ctx *, void *const *x, int n, const void *v, const void *vhat, const void *gv, double factor);
  int (*gnorm)(spm_ctx *, const void *const *x, int n);
  int (*hisd_step)(spm_ctx *, void *x, const void *t, void *dx, double beta);
  // K gated steps of n instances of one grid size and precision, one launch per pass for all
  int (*grad_steps_group)(spm_ctx *const *ctx, void *const *phi, void *const *uhat, int n, int nsteps);
  // Hessian products before their mean removal; scal: SC_MU = the mean, SC_SUM1 = <v, o>, SC_SUM2 = mean(v)
  int (*hv_raw)(spm_ctx *, const void *phi, const void *const *v, void *const *hv, int n);
};

// prec: 0 = FP64, 1 = FP32
const OpsTable *spm_table_32(int prec);
const OpsTable *spm_table_64(int prec);
const OpsTable *spm_table_96(int prec);
const OpsTable *spm_table_128(int prec);
const OpsTable *spm_table_160(int prec);
const OpsTable *spm_table_192(int prec);
const OpsTable *spm_table_256(int prec);
