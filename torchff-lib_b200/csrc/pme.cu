// PME entry points: plan management and the drop-in pme_long_range (rank 0).
#include "pme.cuh"

namespace tff {

int pme_cufft_fail(cufftResult r, const char *what) {
  set_error("cuFFT error %d in %s", (int)r, what);
  return TFF_ERR_CUFFT;
}

namespace {

template <class T>
int pme_long_range_impl(const PmePlanImpl &p, int64_t n, const T *x, const T *box, const T *q, double alpha,
                        const T *xm, const T *ym, const T *zm, T *energy, T *phi, T *grad, void *ws, size_t ws_bytes,
                        cudaStream_t s) {
  PmeLayout L = pme_layout(p.dtype, p.K);
  if (ws == nullptr || ws_bytes < L.bytes) {
    set_error("workspace too small: need %zu bytes, got %zu", L.bytes, ws_bytes);
    return TFF_ERR_WORKSPACE;
  }
  char *w = static_cast<char *>(ws);
  PlainAtoms<T> atoms{x, q, n};
  T *phi_grid = nullptr;
  int st = pme_grid_phase<T>(p, L, w, atoms, n, box, alpha, xm, ym, zm, s, &phi_grid);
  if (st != TFF_OK) return st;
  if (n == 0) {
    // no atoms: energy is the (zero) reciprocal sum
    TFF_CUDA(cudaMemsetAsync(energy, 0, sizeof(T), s));
    return TFF_OK;
  }
  PlainGatherOut<T> out{phi, grad};
  return pme_gather_phase<T>(p, L, w, atoms, n, box, alpha, phi_grid, out, 1.0, energy, s);
}

}  // namespace
}  // namespace tff

using namespace tff;

extern "C" {

int tff_pme_plan_create(int dtype, int K, tff_pme_plan *plan) {
  TFF_ARG(dtype == TFF_F32 || dtype == TFF_F64, "dtype must be TFF_F32 or TFF_F64");
  TFF_ARG(K >= 6 && K <= 1024, "PME grid K must be in [6, 1024] (order-6 splines)");
  TFF_ARG(plan != nullptr, "plan is NULL");
  auto *p = new tff_pme_plan_s();
  p->impl.dtype = dtype;
  p->impl.K = K;
  cudaGetDevice(&p->impl.device);
  cufftResult r = cufftPlan3d(&p->impl.r2c, K, K, K, dtype == TFF_F64 ? CUFFT_D2Z : CUFFT_R2C);
  if (r != CUFFT_SUCCESS) {
    delete p;
    return pme_cufft_fail(r, "cufftPlan3d(R2C)");
  }
  r = cufftPlan3d(&p->impl.c2r, K, K, K, dtype == TFF_F64 ? CUFFT_Z2D : CUFFT_C2R);
  if (r != CUFFT_SUCCESS) {
    cufftDestroy(p->impl.r2c);
    delete p;
    return pme_cufft_fail(r, "cufftPlan3d(C2R)");
  }
  *plan = p;
  return TFF_OK;
}

int tff_pme_plan_destroy(tff_pme_plan plan) {
  if (!plan) return TFF_OK;
  cufftDestroy(plan->impl.r2c);
  cufftDestroy(plan->impl.c2r);
  delete plan;
  return TFF_OK;
}

size_t tff_pme_workspace_bytes(tff_pme_plan plan, int64_t natoms) {
  (void)natoms;
  if (!plan) return 0;
  return pme_layout(plan->impl.dtype, plan->impl.K).bytes;
}

int tff_pme_long_range(tff_pme_plan plan, int64_t natoms, const void *coords, const void *box, const void *charges,
                       double alpha, const void *xmoduli, const void *ymoduli, const void *zmoduli, void *energy,
                       void *phi, void *grad_coords, void *workspace, size_t workspace_bytes, tff_stream_t stream) {
  TFF_NVTX("tff_pme_long_range");
  TFF_ARG(plan != nullptr, "plan is NULL");
  TFF_ARG(natoms >= 0, "negative natoms");
  TFF_ARG(box != nullptr, "PME requires a periodic box");
  TFF_ARG(energy != nullptr, "energy is NULL");
  TFF_ARG(natoms == 0 || (coords != nullptr && charges != nullptr), "coords/charges is NULL");
  TFF_ARG(xmoduli && ymoduli && zmoduli, "B-spline moduli are NULL");
  TFF_ARG(alpha > 0.0, "alpha must be positive");
  cudaStream_t s = (cudaStream_t)stream;
  if (plan->impl.dtype == TFF_F32)
    return pme_long_range_impl<float>(plan->impl, natoms, (const float *)coords, (const float *)box,
                                      (const float *)charges, alpha, (const float *)xmoduli, (const float *)ymoduli,
                                      (const float *)zmoduli, (float *)energy, (float *)phi, (float *)grad_coords,
                                      workspace, workspace_bytes, s);
  return pme_long_range_impl<double>(plan->impl, natoms, (const double *)coords, (const double *)box,
                                     (const double *)charges, alpha, (const double *)xmoduli, (const double *)ymoduli,
                                     (const double *)zmoduli, (double *)energy, (double *)phi, (double *)grad_coords,
                                     workspace, workspace_bytes, s);
}

}  // extern "C"
