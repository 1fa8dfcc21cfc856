// extern "C" entry points of libairt (declared in include/airt.h).  Each one
// converts C++ exceptions into a status code plus a thread-local message.
#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <mutex>

#include <vector>

#include "common.cuh"

namespace airt {

static thread_local std::string g_last_error;

void set_error(const char *fmt, ...) {
  char buf[1024];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  g_last_error = buf;
}

void prof_begin(Problem &P, int which, cudaEvent_t *ev0) {
  (void)which;
  *ev0 = nullptr;
  if (!P.profiling) return;
  cudaEvent_t e;
  if (P.ev_pool.empty()) {
    AIRT_CHECK_CUDA(cudaEventCreate(&e));
  } else {
    e = P.ev_pool.back();
    P.ev_pool.pop_back();
  }
  AIRT_CHECK_CUDA(cudaEventRecord(e, P.stream));
  *ev0 = e;
}

void prof_end(Problem &P, int which, cudaEvent_t ev0) {
  if (!P.profiling || !ev0) return;
  cudaEvent_t e;
  if (P.ev_pool.empty()) {
    AIRT_CHECK_CUDA(cudaEventCreate(&e));
  } else {
    e = P.ev_pool.back();
    P.ev_pool.pop_back();
  }
  AIRT_CHECK_CUDA(cudaEventRecord(e, P.stream));
  P.ev_pending.push_back({which, {ev0, e}});
}

void prof_collect(Problem &P) {
  if (P.ev_pending.empty()) return;
  AIRT_CHECK_CUDA(cudaStreamSynchronize(P.stream));
  for (auto &it : P.ev_pending) {
    float ms = 0;
    cudaEventElapsedTime(&ms, it.second.first, it.second.second);
    P.prof_ms[it.first] += ms;
    P.prof_launches[it.first] += 1;
    P.ev_pool.push_back(it.second.first);
    P.ev_pool.push_back(it.second.second);
  }
  P.ev_pending.clear();
}

static Problem *new_problem() {
  Problem *P = new Problem();
  const char *kind = getenv("AIRT_SPMV");
  P->spmv_kind = (kind && strcmp(kind, "stream") == 0) ? 1 : 0;
  cudaError_t e = cudaStreamCreateWithFlags(&P->stream, cudaStreamNonBlocking);
  if (e != cudaSuccess) {
    delete P;
    set_error("cudaStreamCreate failed: %s", cudaGetErrorString(e));
    throw Status{AIRT_ERR_CUDA};
  }
  return P;
}

static void free_problem(Problem *P) {
  if (!P) return;
  if (P->stream) cudaStreamSynchronize(P->stream);
  for (auto &it : P->ev_pending) {
    cudaEventDestroy(it.second.first);
    cudaEventDestroy(it.second.second);
  }
  for (auto e : P->ev_pool) cudaEventDestroy(e);
  if (P->h_state) cudaFreeHost(P->h_state);
  cudaStream_t s = P->stream;
  delete P;
  if (s) cudaStreamDestroy(s);
}

}  // namespace airt

using namespace airt;

namespace airt {
int g_alloc_fail_countdown = -1;
}

#define AIRT_API_BEGIN try {
#define AIRT_API_END                                   \
  }                                                    \
  catch (const airt::Status &st) {                     \
    return st.code;                                    \
  }                                                    \
  catch (const std::bad_alloc &) {                     \
    airt::set_error("host allocation failed");         \
    return AIRT_ERR_OOM;                               \
  }                                                    \
  catch (...) {                                        \
    airt::set_error("unexpected internal error");      \
    return AIRT_ERR_CUDA;                              \
  }                                                    \
  return AIRT_OK;

extern "C" {

const char *airt_last_error(void) { return g_last_error.c_str(); }

int airt_version(void) { return 10000; }

int airt_problem_from_csc(int64_t m, int64_t n, const uint64_t *jc, const uint64_t *ir,
                          const double *pr, airt_problem **out) {
  AIRT_API_BEGIN
  AIRT_REQUIRE(out && jc, "null pointer argument");
  AIRT_REQUIRE(m >= 0 && n >= 0 && m < INT32_MAX && n < INT32_MAX, "matrix size out of range");
  const int64_t nnz = (int64_t)jc[n];
  AIRT_REQUIRE(jc[0] == 0, "jc[0] must be 0");
  for (int64_t j = 0; j < n; ++j) AIRT_REQUIRE(jc[j + 1] >= jc[j], "jc must be nondecreasing");
  AIRT_REQUIRE(nnz == 0 || (ir && pr), "null pointer argument");
  Problem *P = new_problem();
  try {
    P->m = m;
    P->n = n;
    P->nnz = nnz;
    build_csr_from_host_csc(*P, jc, ir, pr);
    finalize_matrix(*P);
  } catch (...) {
    free_problem(P);
    throw;
  }
  *out = reinterpret_cast<airt_problem *>(P);
  AIRT_API_END
}

static int make_geometry(int kind, int N, int nA, const double *cos_t, const double *sin_t, int p,
                         const double *offsets, const double *cos_w, const double *sin_w, double R,
                         int matrix_free, airt_problem **out) {
  AIRT_API_BEGIN
  AIRT_REQUIRE(out && cos_t && sin_t, "null pointer argument");
  AIRT_REQUIRE(N >= 1 && N <= 46340 && nA >= 0 && p >= 0, "geometry size out of range");
  AIRT_REQUIRE((int64_t)nA * p < INT32_MAX, "too many rays");
  Problem *P = new_problem();
  try {
    P->geo_kind = kind;
    P->N = N;
    P->nA = nA;
    P->p = p;
    P->R = R;
    P->m = (int64_t)nA * p;
    P->n = (int64_t)N * N;
    P->matrix_free = matrix_free != 0;
    P->cos_t.upload(cos_t, nA, P->stream);
    P->sin_t.upload(sin_t, nA, P->stream);
    if (kind == GEO_PARALLEL) {
      AIRT_REQUIRE(offsets || p == 0, "null pointer argument");
      P->offsets.upload(offsets, p, P->stream);
    } else {
      AIRT_REQUIRE((cos_w && sin_w) || p == 0, "null pointer argument");
      AIRT_REQUIRE(R >= std::sqrt(2.0) / 2.0 * N, "R must be greater than half squareroot 2");
      P->cos_w.upload(cos_w, p, P->stream);
      P->sin_w.upload(sin_w, p, P->stream);
    }
    AIRT_CHECK_CUDA(cudaStreamSynchronize(P->stream));
    if (!P->matrix_free) generate_matrix(*P);
    else mf_prepare(*P);
  } catch (...) {
    free_problem(P);
    throw;
  }
  *out = reinterpret_cast<airt_problem *>(P);
  AIRT_API_END
}

int airt_problem_parallel(int N, int nA, const double *cos_t, const double *sin_t, int p,
                          const double *offsets, int matrix_free, airt_problem **out) {
  return make_geometry(GEO_PARALLEL, N, nA, cos_t, sin_t, p, offsets, nullptr, nullptr, 0.0,
                       matrix_free, out);
}

int airt_problem_fan(int N, int nA, const double *cos_t, const double *sin_t, int p,
                     const double *cos_w, const double *sin_w, double R, int matrix_free,
                     airt_problem **out) {
  return make_geometry(GEO_FAN, N, nA, cos_t, sin_t, p, nullptr, cos_w, sin_w, R, matrix_free, out);
}

int airt_problem_seismic(int N, int s, const double *src_x, const double *src_y, int p,
                         const double *rcv_x, const double *rcv_y, int matrix_free,
                         airt_problem **out) {
  AIRT_API_BEGIN
  AIRT_REQUIRE(out, "null pointer argument");
  AIRT_REQUIRE((src_x && src_y) || s == 0, "null pointer argument");
  AIRT_REQUIRE((rcv_x && rcv_y) || p == 0, "null pointer argument");
  AIRT_REQUIRE(N >= 1 && N <= 46340 && s >= 0 && p >= 0, "geometry size out of range");
  AIRT_REQUIRE((int64_t)s * p < INT32_MAX, "too many rays");
  Problem *P = new_problem();
  try {
    P->geo_kind = GEO_SEISMIC;
    P->N = N;
    P->nA = s;
    P->p = p;
    P->m = (int64_t)s * p;
    P->n = (int64_t)N * N;
    P->matrix_free = matrix_free != 0;
    P->src_x.upload(src_x, s, P->stream);
    P->src_y.upload(src_y, s, P->stream);
    P->rcv_x.upload(rcv_x, p, P->stream);
    P->rcv_y.upload(rcv_y, p, P->stream);
    AIRT_CHECK_CUDA(cudaStreamSynchronize(P->stream));
    if (!P->matrix_free) generate_matrix(*P);
    else mf_prepare(*P);
  } catch (...) {
    free_problem(P);
    throw;
  }
  *out = reinterpret_cast<airt_problem *>(P);
  AIRT_API_END
}

int airt_problem_spherical(int N, int nA, const double *cos_t, const double *sin_t, int nc,
                           const double *radius, const int64_t *nphi, const double *cos_k,
                           const double *sin_k, int matrix_free, airt_problem **out) {
  AIRT_API_BEGIN
  AIRT_REQUIRE(out, "null pointer argument");
  AIRT_REQUIRE((cos_t && sin_t) || nA == 0, "null pointer argument");
  AIRT_REQUIRE((radius && nphi) || nc == 0, "null pointer argument");
  AIRT_REQUIRE(N >= 1 && N <= 46340 && nA >= 0 && nc >= 0, "geometry size out of range");
  AIRT_REQUIRE((int64_t)nA * nc < INT32_MAX, "too many rows");
  std::vector<int64_t> koff(nc + 1, 0);
  std::vector<double> cscale(nc);
  for (int n = 0; n < nc; ++n) {
    AIRT_REQUIRE(nphi[n] >= 1, "nphi must be positive");
    koff[n + 1] = koff[n] + nphi[n] + 1;  // k = (0:nPhi)*dPhi, sphericaltomo.m:203
    // 2*pi*radii(n)/nPhi(n), sphericaltomo.m:234
    cscale[n] = 2.0 * 3.141592653589793 * radius[n] / (double)nphi[n];
  }
  AIRT_REQUIRE(koff[nc] < INT32_MAX, "too many samples per angle");
  AIRT_REQUIRE(koff[nc] == 0 || (cos_k && sin_k), "null pointer argument");
  Problem *P = new_problem();
  try {
    P->geo_kind = GEO_SPHERE;
    P->N = N;
    P->nA = nA;
    P->p = nc;
    P->m = (int64_t)nA * nc;
    P->n = (int64_t)N * N;
    P->matrix_free = matrix_free != 0;
    P->dx = std::sqrt(2.0) / N;           // sphericaltomo.m:122
    P->center = (N + 1) / 2;              // ceil(N/2), sphericaltomo.m:119
    P->koff_total = koff[nc];
    P->cos_t.upload(cos_t, nA, P->stream);
    P->sin_t.upload(sin_t, nA, P->stream);
    P->radius.upload(radius, nc, P->stream);
    P->cscale.upload(cscale.data(), nc, P->stream);
    P->koff.upload(koff.data(), nc + 1, P->stream);
    P->cos_k.upload(cos_k, koff[nc], P->stream);
    P->sin_k.upload(sin_k, koff[nc], P->stream);
    AIRT_CHECK_CUDA(cudaStreamSynchronize(P->stream));
    if (!P->matrix_free) generate_matrix(*P);
    else mf_prepare(*P);
  } catch (...) {
    free_problem(P);
    throw;
  }
  *out = reinterpret_cast<airt_problem *>(P);
  AIRT_API_END
}

int airt_problem_size(const airt_problem *h, int64_t *m, int64_t *n, int64_t *nnz) {
  AIRT_API_BEGIN
  AIRT_REQUIRE(h, "null problem handle");
  const Problem *P = reinterpret_cast<const Problem *>(h);
  if (m) *m = P->m;
  if (n) *n = P->n;
  if (nnz) *nnz = P->matrix_free ? -1 : P->nnz;
  AIRT_API_END
}

int airt_problem_stream(const airt_problem *h, void **cuda_stream) {
  AIRT_API_BEGIN
  AIRT_REQUIRE(h && cuda_stream, "null pointer argument");
  *cuda_stream = (void *)reinterpret_cast<const Problem *>(h)->stream;
  AIRT_API_END
}

int airt_problem_export_csc(airt_problem *h, uint64_t *jc, uint64_t *ir, double *pr) {
  AIRT_API_BEGIN
  AIRT_REQUIRE(h && jc, "null pointer argument");
  Problem *P = reinterpret_cast<Problem *>(h);
  AIRT_REQUIRE(P->nnz == 0 || (ir && pr), "null pointer argument");
  export_csc(*P, jc, ir, pr);
  AIRT_API_END
}

int airt_destroy(airt_problem *h) {
  AIRT_API_BEGIN
  free_problem(reinterpret_cast<Problem *>(h));
  AIRT_API_END
}

int airt_apply(airt_problem *h, const double *in, double *out, int transp) {
  AIRT_API_BEGIN
  AIRT_REQUIRE(h && in && out, "null pointer argument");
  Problem *P = reinterpret_cast<Problem *>(h);
  const int64_t nin = transp ? P->m : P->n, nout = transp ? P->n : P->m;
  P->vin.upload(in, nin, P->stream);
  P->vout.ensure(nout);
  apply_operator(*P, P->vin.p, P->vout.p, transp);
  AIRT_CHECK_CUDA(cudaMemcpyAsync(out, P->vout.p, nout * sizeof(double), cudaMemcpyDeviceToHost,
                                  P->stream));
  AIRT_CHECK_CUDA(cudaStreamSynchronize(P->stream));
  AIRT_API_END
}

int airt_apply_device(airt_problem *h, const double *d_in, double *d_out, int transp) {
  AIRT_API_BEGIN
  AIRT_REQUIRE(h && d_in && d_out, "null pointer argument");
  Problem *P = reinterpret_cast<Problem *>(h);
  apply_operator(*P, d_in, d_out, transp);
  AIRT_API_END
}

int airt_weights(airt_problem *h, int method, double *M, double *D) {
  AIRT_API_BEGIN
  AIRT_REQUIRE(h && M && D, "null pointer argument");
  AIRT_REQUIRE(method >= AIRT_LANDWEBER && method <= AIRT_SART, "SIRT method not defined.");
  Problem *P = reinterpret_cast<Problem *>(h);
  P->M.ensure(P->m);
  P->D.ensure(P->n);
  compute_weights(*P, method, P->M.p, P->D.p);
  AIRT_CHECK_CUDA(cudaMemcpyAsync(M, P->M.p, P->m * sizeof(double), cudaMemcpyDeviceToHost, P->stream));
  AIRT_CHECK_CUDA(cudaMemcpyAsync(D, P->D.p, P->n * sizeof(double), cudaMemcpyDeviceToHost, P->stream));
  AIRT_CHECK_CUDA(cudaStreamSynchronize(P->stream));
  AIRT_API_END
}

int airt_rho(airt_problem *h, int method, const double *Mcustom, const double *Dcustom, double tol,
             int maxit, double *rho) {
  AIRT_API_BEGIN
  AIRT_REQUIRE(h && rho, "null pointer argument");
  AIRT_REQUIRE(maxit > 0 && tol >= 0, "invalid tolerance or iteration limit");
  Problem *P = reinterpret_cast<Problem *>(h);
  P->M.ensure(P->m);
  P->D.ensure(P->n);
  if (method == AIRT_CUSTOM) {
    std::vector<double> ones;
    if (Mcustom) P->M.upload(Mcustom, P->m, P->stream);
    else {
      ones.assign(P->m, 1.0);
      P->M.upload(ones.data(), P->m, P->stream);
    }
    if (Dcustom) P->D.upload(Dcustom, P->n, P->stream);
    else {
      ones.assign(P->n, 1.0);
      P->D.upload(ones.data(), P->n, P->stream);
    }
    AIRT_CHECK_CUDA(cudaStreamSynchronize(P->stream));
  } else {
    AIRT_REQUIRE(method >= AIRT_LANDWEBER && method <= AIRT_SART, "SIRT method not defined.");
    compute_weights(*P, method, P->M.p, P->D.p);
  }
  *rho = estimate_rho(*P, P->M.p, P->D.p, tol, maxit);
  AIRT_API_END
}

int airt_sirt_multi_device(airt_problem *h, const airt_sirt_opts *opts, int K, const double *d_B,
                           const double *d_X0, const double *taudelta, const double *relaxpar,
                           const int64_t *Ksave, int64_t nsave, double *d_Xsave, double *d_X,
                           int64_t *finaliter, int *stoprule, double *gpu_ms) {
  AIRT_API_BEGIN
  AIRT_REQUIRE(h && opts && d_B && d_X, "null pointer argument");
  run_sirt_multi(*reinterpret_cast<Problem *>(h), *opts, K, d_B, d_X0, taudelta, relaxpar, Ksave,
                 nsave, d_Xsave, d_X, finaliter, stoprule, gpu_ms);
  AIRT_API_END
}

int airt_rho_custom(airt_problem *h, const double *M, int M_full, const double *D, int D_full,
                    double tol, int maxit, double *rho) {
  AIRT_API_BEGIN
  AIRT_REQUIRE(h && rho, "null pointer argument");
  AIRT_REQUIRE(maxit > 0 && tol >= 0, "invalid tolerance or iteration limit");
  Problem *P = reinterpret_cast<Problem *>(h);
  const bool mf = M && M_full, df = D && D_full;
  AIRT_REQUIRE(!mf || (double)P->m * (double)P->m <= 4e9, "a full custom M does not fit the device");
  AIRT_REQUIRE(!df || (double)P->n * (double)P->n <= 4e9, "a full custom D does not fit the device");
  const double *dM = nullptr, *dD = nullptr;
  if (mf) {
    P->Mfull.upload(M, (size_t)P->m * P->m, P->stream);
    dM = P->Mfull.p;
  } else if (M) {
    P->M.upload(M, P->m, P->stream);
    dM = P->M.p;
  }
  if (df) {
    P->Dfull.upload(D, (size_t)P->n * P->n, P->stream);
    dD = P->Dfull.p;
  } else if (D) {
    P->D.upload(D, P->n, P->stream);
    dD = P->D.p;
  }
  *rho = estimate_rho_custom(*P, dM, mf, dD, df, tol, maxit);
  AIRT_API_END
}

int airt_sirt_device(airt_problem *h, const airt_sirt_opts *opts, const double *d_b,
                     const double *d_x0, const int64_t *K, int64_t nK, double *d_X,
                     double *resnorms, airt_info *info) {
  AIRT_API_BEGIN
  AIRT_REQUIRE(h && opts && d_b && d_X, "null pointer argument");
  Problem *P = reinterpret_cast<Problem *>(h);
  run_sirt(*P, *opts, d_b, d_x0, K, nK, d_X, resnorms, info);
  AIRT_API_END
}

int airt_sirt(airt_problem *h, const airt_sirt_opts *opts, const double *b, const double *x0,
              const int64_t *K, int64_t nK, double *X, double *resnorms, airt_info *info) {
  AIRT_API_BEGIN
  AIRT_REQUIRE(h && opts && b && X, "null pointer argument");
  Problem *P = reinterpret_cast<Problem *>(h);
  cudaStream_t s = P->stream;
  P->b64.upload(b, P->m, s);
  if (x0) P->vin.upload(x0, P->n, s);
  P->Xd.ensure((size_t)P->n * (nK > 0 ? nK : 1));
  airt_info inf{};
  run_sirt(*P, *opts, P->b64.p, x0 ? P->vin.p : nullptr, K, nK, P->Xd.p, resnorms, &inf);
  if (inf.nsaved)
    AIRT_CHECK_CUDA(cudaMemcpyAsync(X, P->Xd.p, (size_t)inf.nsaved * P->n * sizeof(double),
                                    cudaMemcpyDeviceToHost, s));
  AIRT_CHECK_CUDA(cudaStreamSynchronize(s));
  if (info) *info = inf;
  AIRT_API_END
}

int airt_art(airt_problem *h, const airt_art_opts *opts, const double *b, const double *x0,
             const int64_t *K, int64_t nK, double *X, double *resnorms, airt_info *info) {
  AIRT_API_BEGIN
  AIRT_REQUIRE(h && opts && b && X, "null pointer argument");
  Problem *P = reinterpret_cast<Problem *>(h);
  cudaStream_t s = P->stream;
  P->b64.upload(b, P->m, s);
  if (x0) P->vin.upload(x0, P->n, s);
  P->Xd.ensure((size_t)P->n * (nK > 0 ? nK : 1));
  airt_info inf{};
  run_art(*P, *opts, P->b64.p, x0 ? P->vin.p : nullptr, K, nK, P->Xd.p, resnorms, &inf);
  if (inf.nsaved)
    AIRT_CHECK_CUDA(cudaMemcpyAsync(X, P->Xd.p, (size_t)inf.nsaved * P->n * sizeof(double),
                                    cudaMemcpyDeviceToHost, s));
  AIRT_CHECK_CUDA(cudaStreamSynchronize(s));
  if (info) *info = inf;
  AIRT_API_END
}

int airt_cart(airt_problem *h, const airt_cart_opts *opts, const double *b, const double *x0,
              const int64_t *K, int64_t nK, double *X, double *resnorms, airt_info *info) {
  AIRT_API_BEGIN
  AIRT_REQUIRE(h && opts && b && X, "null pointer argument");
  Problem *P = reinterpret_cast<Problem *>(h);
  cudaStream_t s = P->stream;
  P->b64.upload(b, P->m, s);
  if (x0) P->vin.upload(x0, P->n, s);
  P->Xd.ensure((size_t)P->n * (nK > 0 ? nK : 1));
  airt_info inf{};
  run_cart(*P, *opts, P->b64.p, x0 ? P->vin.p : nullptr, K, nK, P->Xd.p, resnorms, &inf);
  if (inf.nsaved)
    AIRT_CHECK_CUDA(cudaMemcpyAsync(X, P->Xd.p, (size_t)inf.nsaved * P->n * sizeof(double),
                                    cudaMemcpyDeviceToHost, s));
  AIRT_CHECK_CUDA(cudaStreamSynchronize(s));
  if (info) *info = inf;
  AIRT_API_END
}

// ---------------------------------------------------------------- batches
int airt_batch_parallel(int ninst, const int *N, const int *nA, const int *p, const double *cos_t,
                        const double *sin_t, const double *offsets, airt_batch **out) {
  AIRT_API_BEGIN
  AIRT_REQUIRE(out && N && nA && p && cos_t && sin_t && offsets && ninst >= 1,
               "null pointer argument or empty batch");
  *out = reinterpret_cast<airt_batch *>(batch_build(ninst, N, nA, p, cos_t, sin_t, offsets));
  AIRT_API_END
}

int airt_batch_layout(const airt_batch *h, int64_t *row_off, int64_t *col_off, int64_t *nnz) {
  AIRT_API_BEGIN
  AIRT_REQUIRE(h, "null batch handle");
  Batch &B = *reinterpret_cast<Batch *>(const_cast<airt_batch *>(h));
  const int K = batch_ninst(B);
  if (row_off) std::copy(batch_row_off(B), batch_row_off(B) + K + 1, row_off);
  if (col_off) std::copy(batch_col_off(B), batch_col_off(B) + K + 1, col_off);
  if (nnz) *nnz = batch_problem(B).nnz;
  AIRT_API_END
}

int airt_batch_stream(const airt_batch *h, void **cuda_stream) {
  AIRT_API_BEGIN
  AIRT_REQUIRE(h && cuda_stream, "null pointer argument");
  Batch &B = *reinterpret_cast<Batch *>(const_cast<airt_batch *>(h));
  *cuda_stream = (void *)batch_problem(B).stream;
  AIRT_API_END
}

int airt_batch_rho(airt_batch *h, int method, double tol, int maxit, double *rho) {
  AIRT_API_BEGIN
  AIRT_REQUIRE(h && rho && maxit > 0, "invalid argument");
  AIRT_REQUIRE(method >= AIRT_LANDWEBER && method <= AIRT_SART, "SIRT method not defined.");
  batch_rho(*reinterpret_cast<Batch *>(h), method, tol, maxit, rho);
  AIRT_API_END
}

int airt_batch_sirt_device(airt_batch *h, int method, const double *relaxpar, const double *d_b,
                           const double *taudelta, int64_t kmax, int lb_kind, double lb, int ub_kind,
                           double ub, const double *d_x0, double *d_x, int64_t *finaliter,
                           int *stoprule, double *gpu_ms) {
  AIRT_API_BEGIN
  AIRT_REQUIRE(h && relaxpar && d_b && d_x, "null pointer argument");
  AIRT_REQUIRE(method >= AIRT_LANDWEBER && method <= AIRT_SART, "SIRT method not defined.");
  AIRT_REQUIRE(lb_kind != AIRT_BOUND_VECTOR && ub_kind != AIRT_BOUND_VECTOR,
               "batched SIRT takes scalar bounds");
  batch_sirt(*reinterpret_cast<Batch *>(h), method, relaxpar, d_b,
             taudelta ? AIRT_STOP_DP : AIRT_STOP_NONE, taudelta, 2, kmax, lb_kind, lb, ub_kind, ub,
             d_x0, d_x, finaliter, stoprule, gpu_ms);
  AIRT_API_END
}

int airt_batch_sirt(airt_batch *h, int method, const double *relaxpar, const double *b,
                    const double *taudelta, int64_t kmax, int lb_kind, double lb, int ub_kind,
                    double ub, const double *x0, double *x, int64_t *finaliter, int *stoprule,
                    double *gpu_ms) {
  AIRT_API_BEGIN
  AIRT_REQUIRE(h && relaxpar && b && x, "null pointer argument");
  Batch &B = *reinterpret_cast<Batch *>(h);
  Problem &P = batch_problem(B);
  P.b64.upload(b, P.m, P.stream);
  if (x0) P.vin.upload(x0, P.n, P.stream);
  P.Xd.ensure(P.n);
  AIRT_REQUIRE(method >= AIRT_LANDWEBER && method <= AIRT_SART, "SIRT method not defined.");
  AIRT_REQUIRE(lb_kind != AIRT_BOUND_VECTOR && ub_kind != AIRT_BOUND_VECTOR,
               "batched SIRT takes scalar bounds");
  batch_sirt(B, method, relaxpar, P.b64.p, taudelta ? AIRT_STOP_DP : AIRT_STOP_NONE, taudelta, 2,
             kmax, lb_kind, lb, ub_kind, ub, x0 ? P.vin.p : nullptr, P.Xd.p, finaliter, stoprule,
             gpu_ms);
  AIRT_CHECK_CUDA(cudaMemcpyAsync(x, P.Xd.p, P.n * sizeof(double), cudaMemcpyDeviceToHost, P.stream));
  AIRT_CHECK_CUDA(cudaStreamSynchronize(P.stream));
  AIRT_API_END
}

int airt_batch_sirt_rule(airt_batch *h, int method, const double *relaxpar, const double *b,
                         int stoprule, const double *taudelta, int ncp_smooth, int64_t kmax,
                         int lb_kind, double lb, int ub_kind, double ub, const double *x0, double *x,
                         int64_t *finaliter, int *stoprule_out, double *gpu_ms) {
  AIRT_API_BEGIN
  AIRT_REQUIRE(h && relaxpar && b && x, "null pointer argument");
  Batch &B = *reinterpret_cast<Batch *>(h);
  Problem &P = batch_problem(B);
  AIRT_REQUIRE(method >= AIRT_LANDWEBER && method <= AIRT_SART, "SIRT method not defined.");
  AIRT_REQUIRE(lb_kind != AIRT_BOUND_VECTOR && ub_kind != AIRT_BOUND_VECTOR,
               "batched SIRT takes scalar bounds");
  P.b64.upload(b, P.m, P.stream);
  if (x0) P.vin.upload(x0, P.n, P.stream);
  P.Xd.ensure(P.n);
  batch_sirt(B, method, relaxpar, P.b64.p, stoprule, taudelta, ncp_smooth, kmax, lb_kind, lb,
             ub_kind, ub, x0 ? P.vin.p : nullptr, P.Xd.p, finaliter, stoprule_out, gpu_ms);
  AIRT_CHECK_CUDA(cudaMemcpyAsync(x, P.Xd.p, P.n * sizeof(double), cudaMemcpyDeviceToHost, P.stream));
  AIRT_CHECK_CUDA(cudaStreamSynchronize(P.stream));
  AIRT_API_END
}

int airt_batch_nnz(const airt_batch *h, int64_t *nnz) {
  AIRT_API_BEGIN
  AIRT_REQUIRE(h && nnz, "null pointer argument");
  Batch &B = *reinterpret_cast<Batch *>(const_cast<airt_batch *>(h));
  Problem &P = batch_problem(B);
  const int K = batch_ninst(B);
  const int64_t *roff = batch_row_off(B);
  std::vector<int64_t> ptr(K + 1);
  for (int k = 0; k <= K; ++k)
    AIRT_CHECK_CUDA(cudaMemcpy(&ptr[k], P.rp.p + roff[k], sizeof(int64_t), cudaMemcpyDeviceToHost));
  for (int k = 0; k < K; ++k) nnz[k] = ptr[k + 1] - ptr[k];
  AIRT_API_END
}

int airt_batch_apply(airt_batch *h, const double *d_in, double *d_out, int transp) {
  AIRT_API_BEGIN
  AIRT_REQUIRE(h && d_in && d_out, "null pointer argument");
  Problem &P = batch_problem(*reinterpret_cast<Batch *>(h));
  apply_operator(P, d_in, d_out, transp);
  AIRT_CHECK_CUDA(cudaStreamSynchronize(P.stream));
  AIRT_API_END
}

int airt_batch_backproject(airt_batch *h, int method, const double *d_b, double *d_x, double *gpu_ms) {
  AIRT_API_BEGIN
  AIRT_REQUIRE(h && d_b && d_x, "null pointer argument");
  AIRT_REQUIRE(method >= AIRT_LANDWEBER && method <= AIRT_SART, "SIRT method not defined.");
  batch_backproject(*reinterpret_cast<Batch *>(h), method, d_b, d_x, gpu_ms);
  AIRT_API_END
}

int airt_fbp(airt_problem *h, const double *b, int na, const double *kernel, int order,
                        double *x) {
  AIRT_API_BEGIN
  AIRT_REQUIRE(h && b && kernel && x, "null pointer argument");
  Problem *P = reinterpret_cast<Problem *>(h);
  AIRT_REQUIRE(na >= 1 && P->m % na == 0, "fbp: the number of angles must divide the rows of A");
  const int64_t nr64 = P->m / na;
  AIRT_REQUIRE(nr64 >= 1 && nr64 < INT32_MAX, "fbp: projection length out of range");
  const int nr = (int)nr64;
  cudaStream_t s = P->stream;
  P->fbp_h.upload(kernel, order, s);
  P->b64.upload(b, P->m, s);
  P->fbp_tmp.ensure(P->m);
  const double scale = 3.141592653589793 / (2.0 * na);  // fbp.m:79
  fbp_filter(P->b64.p, P->fbp_tmp.p, nr, na, P->fbp_h.p, order, nullptr, scale, s);
  P->vout.ensure(P->n);
  apply_operator(*P, P->fbp_tmp.p, P->vout.p, 1);
  AIRT_CHECK_CUDA(cudaMemcpyAsync(x, P->vout.p, P->n * sizeof(double), cudaMemcpyDeviceToHost, s));
  AIRT_CHECK_CUDA(cudaStreamSynchronize(s));
  AIRT_API_END
}

int airt_batch_fbp(airt_batch *h, const double *d_b, int nr, const double *kernel,
                              int order, const double *col_scale, double *d_x, double *gpu_ms) {
  AIRT_API_BEGIN
  AIRT_REQUIRE(h && d_b && kernel && col_scale && d_x, "null pointer argument");
  Batch &B = *reinterpret_cast<Batch *>(h);
  Problem &P = batch_problem(B);
  const int K = batch_ninst(B);
  const int64_t *roff = batch_row_off(B);
  for (int k = 0; k < K; ++k)
    AIRT_REQUIRE(nr >= 1 && (roff[k + 1] - roff[k]) % nr == 0,
                 "batch fbp: every instance needs projections of nr rays");
  const int64_t ncols = P.m / nr;
  cudaStream_t s = P.stream;
  cudaEvent_t t0, t1;
  AIRT_CHECK_CUDA(cudaEventCreate(&t0));
  AIRT_CHECK_CUDA(cudaEventCreate(&t1));
  P.fbp_h.upload(kernel, order, s);
  P.fbp_scale.upload(col_scale, ncols, s);
  P.fbp_tmp.ensure(std::max<int64_t>(P.m, 1));
  AIRT_CHECK_CUDA(cudaEventRecord(t0, s));
  fbp_filter(d_b, P.fbp_tmp.p, nr, ncols, P.fbp_h.p, order, P.fbp_scale.p, 1.0, s);
  apply_operator(P, P.fbp_tmp.p, d_x, 1);
  AIRT_CHECK_CUDA(cudaEventRecord(t1, s));
  AIRT_CHECK_CUDA(cudaStreamSynchronize(s));
  float ms = 0;
  cudaEventElapsedTime(&ms, t0, t1);
  cudaEventDestroy(t0);
  cudaEventDestroy(t1);
  if (gpu_ms) *gpu_ms = ms;
  AIRT_API_END
}

int airt_batch_kaczmarz(airt_batch *h, const double *b, int64_t sweeps, double relaxpar,
                        int lb_kind, double lb, int ub_kind, double ub, double *x, double *gpu_ms) {
  AIRT_API_BEGIN
  AIRT_REQUIRE(h && b && x, "null pointer argument");
  AIRT_REQUIRE(lb_kind != AIRT_BOUND_VECTOR && ub_kind != AIRT_BOUND_VECTOR,
               "batched Kaczmarz takes scalar bounds");
  Batch &B = *reinterpret_cast<Batch *>(h);
  Problem &P = batch_problem(B);
  P.b64.upload(b, P.m, P.stream);
  P.Xd.ensure(P.n);
  batch_kaczmarz(B, P.b64.p, sweeps, relaxpar, lb_kind, lb, ub_kind, ub, P.Xd.p, gpu_ms);
  AIRT_CHECK_CUDA(cudaMemcpyAsync(x, P.Xd.p, P.n * sizeof(double), cudaMemcpyDeviceToHost, P.stream));
  AIRT_CHECK_CUDA(cudaStreamSynchronize(P.stream));
  AIRT_API_END
}

int airt_batch_destroy(airt_batch *h) {
  AIRT_API_BEGIN
  batch_destroy(reinterpret_cast<Batch *>(h));
  AIRT_API_END
}

int airt_profile_enable(airt_problem *h, int on) {
  AIRT_API_BEGIN
  AIRT_REQUIRE(h, "null problem handle");
  Problem *P = reinterpret_cast<Problem *>(h);
  prof_collect(*P);
  P->profiling = on != 0;
  P->prof_launches[0] = P->prof_launches[1] = 0;
  P->prof_ms[0] = P->prof_ms[1] = 0;
  AIRT_API_END
}

int airt_profile_read(airt_problem *h, int which, int64_t *launches, double *total_ms) {
  AIRT_API_BEGIN
  AIRT_REQUIRE(h && which >= 0 && which < 2, "invalid argument");
  Problem *P = reinterpret_cast<Problem *>(h);
  prof_collect(*P);
  if (launches) *launches = P->prof_launches[which];
  if (total_ms) *total_ms = P->prof_ms[which];
  AIRT_API_END
}

}  // extern "C"

extern "C" int airt_test_split_trace(airt_problem *h, int64_t *mismatched, int64_t *split) {
  AIRT_API_BEGIN
  AIRT_REQUIRE(h && mismatched, "null pointer argument");
  Problem *P = reinterpret_cast<Problem *>(h);
  *mismatched = test_split_trace(*P, split);
  AIRT_API_END
}

extern "C" int airt_test_fail_alloc(int after) {
  airt::g_alloc_fail_countdown = after < 0 ? -1 : after;
  return AIRT_OK;
}
