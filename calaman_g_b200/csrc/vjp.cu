// vjp.cu -- the adjoint (vector-Jacobian product) of expm.
//
// For a real loss L(E), E = expm(A), G = dL/dE, the adjoint is
//     Abar = L_g(A^H, G),
// the Frechet derivative at A^H, in direction G, of the function expm
// evaluates for A: g(X) = r_m(X / 2^s)^(2^s) with (m, s) = expm_plan(||A||_1)
// fixed. (For a matrix function with real Taylor coefficients the adjoint of
// L_g(A) is L_g(A^H); the transpose for real types.) This is the convention of
// torch.matrix_exp's backward and equals the upper-right block of
// expm([[A^H, G], [0, A^H]]).
//
// L_g(X, D) is evaluated in forward mode alongside g(X) (Al-Mohy and Higham,
// "Computing the Frechet derivative of the matrix exponential", SIAM J. Matrix
// Anal. Appl. 30(4), 2009, Algorithm 6.4): every product Z = X Y carries
// dZ = dX Y + X dY, the Pade quotient R = Q^-1 P carries
// dR = Q^-1 (dP - dQ R) through the same LU factors, and every squaring carries
// dR <- R dR + dR R. Nothing is stored for a reverse sweep and every GEMM is
// non-transposed; A^H is formed once by a transpose kernel.
//
// Work for m = 13: 19 + 3 s GEMMs, one LU and two n-RHS solves (the forward
// expm is 6 + s GEMMs, one LU and one solve).
#include <utility>

#include "expm_common.cuh"
#include "graph_replay.cuh"

namespace clm {
namespace {

// [Xs | Ds | P0..P_{np-1} | M0..M_{np-1} | T1 | T2 | V | W | LV | LW | LU scratch |
//  (FP32: tensor-core operand parts) | (single tiers: four FP64 n x n squaring buffers)]
template <typename T>
struct VjpWs {
  using Wd = typename Wide<T>::type;
  T *Xs = nullptr, *Ds = nullptr;
  T *P[4] = {nullptr, nullptr, nullptr, nullptr};
  T *M[4] = {nullptr, nullptr, nullptr, nullptr};
  T *T1 = nullptr, *T2 = nullptr, *V = nullptr, *W = nullptr, *LV = nullptr, *LW = nullptr;
  double *norm = nullptr;
  void *lu = nullptr;
  void *tc = nullptr;
  std::size_t tc_bytes = 0;
  void *oz = nullptr;
  std::size_t oz_bytes = 0;
  Wd *wide = nullptr;
  std::size_t carve(void *base, int n, int m, std::size_t ozb) {
    Layout L(base);
    const std::size_t nn = (std::size_t)n * n;
    const int np = pade_num_powers(m);
    Xs = L.take<T>(nn);
    Ds = L.take<T>(nn);
    for (int k = 0; k < np; ++k) P[k] = L.take<T>(nn);
    for (int k = 0; k < np; ++k) M[k] = L.take<T>(nn);
    T1 = L.take<T>(nn);
    T2 = L.take<T>(nn);
    V = L.take<T>(nn);
    W = L.take<T>(nn);
    LV = L.take<T>(nn);
    LW = L.take<T>(nn);
    norm = L.take<double>(1);
    lu = L.take<char>(lu_scratch_bytes(n));
    tc_bytes = tc_scratch_bytes<T>(n);
    if (tc_bytes) tc = L.take<char>(tc_bytes);
    oz_bytes = ozb;
    if (oz_bytes) oz = L.take<char>(oz_bytes);
    if (elem<T>::single) wide = L.take<Wd>(4 * nn);
    return L.used;
  }
};

template <typename T>
std::size_t vjp_bytes(calamanHandle_t h, int n) {
  std::size_t worst = 0;
  for (int m : {3, 5, 7, 9, 13}) {
    VjpWs<T> w;
    worst = std::max(worst, w.carve(nullptr, n, m, oz_scratch_bytes<T>(h, n)));
  }
  return worst;
}

// (R, L) <- (R^2, R L + L R), s times; R, L end in *r, *l (the buffers swap).
template <typename U>
cudaError_t frechet_squarings(cudaStream_t st, int n, int s, U **r, U **l, U **r2, U **l2) {
  for (int k = 0; k < s; ++k) {
    cudaError_t e;
    if ((e = gemm_nn<U>(st, n, n, n, 1.0, *r, n, *l, n, 0.0, *l2, n)) != cudaSuccess) return e;
    if ((e = gemm_nn<U>(st, n, n, n, 1.0, *l, n, *r, n, 1.0, *l2, n)) != cudaSuccess) return e;
    if ((e = gemm_nn<U>(st, n, n, n, 1.0, *r, n, *r, n, 0.0, *r2, n)) != cudaSuccess) return e;
    std::swap(*r, *r2);
    std::swap(*l, *l2);
  }
  return cudaSuccess;
}

template <typename T>
calamanStatus_t vjp_api(calamanHandle_t blas, calamanStream_t stream, int n, const T *A, int lda,
                        const T *G, int ldg, T *gradA, int ldga, T *E, int lde, void *work,
                        std::size_t lwork, int *d_info, calamanExpmPlan_t *plan_out) {
  using R = typename elem<T>::real;
  if (n < 1 || n > kMaxDim || lda < n || ldg < n || ldga < n || (E != nullptr && lde < n) ||
      work == nullptr)
    return blas_status(CALAMAN_STATUS_INVALID_VALUE);
  if (lwork < vjp_bytes<T>(blas, n)) return blas_status(CALAMAN_STATUS_ALLOC_FAILED);
  if (A == nullptr || G == nullptr || gradA == nullptr || d_info == nullptr)
    return blas_status(CALAMAN_STATUS_INVALID_VALUE);
  PointerModeScope pm(blas);
  TimerScope ts(timer_of(blas));
  cudaStream_t st = static_cast<cudaStream_t>(stream);

  // the plan expm(A) uses: ||A||_1 in FP64 on the device, one readback
  VjpWs<T> probe;
  probe.carve(work, n, 13, 0);
  CLM_CUDA(launch_norm1<T>(st, n, A, lda, nullptr, probe.norm));
  double norm = 0.0;
  double *host = (blas && blas->h_pinned) ? blas->h_pinned : &norm;
  CLM_CUDA(cudaMemcpyAsync(host, probe.norm, sizeof(double), cudaMemcpyDeviceToHost, st));
  CLM_CUDA(cudaStreamSynchronize(st));
  norm = *host;
  if (!std::isfinite(norm)) return blas_status(CALAMAN_STATUS_INVALID_VALUE);
  const calamanExpmPlan_t plan = plan_for<R>((R)norm);
  if (plan_out) *plan_out = plan;
  const int m = plan.m, np = pade_num_powers(m);
  const double *b = pade_coeffs(m);

  // everything after the plan: launches only, replayed as a CUDA graph while
  // the configuration repeats
  auto post = [&]() -> calamanStatus_t {
    VjpWs<T> ws;
    ws.carve(work, n, m, oz_scratch_bytes<T>(blas, n));
    GemmScratch gs = lend_scratch<T>(blas, n, ws.tc, ws.tc_bytes, ws.oz, ws.oz_bytes);
    GemmScratchScope gss((ws.tc || ws.oz) ? &gs : nullptr);
    auto mm = [&](const T *X, const T *Y, double beta, T *Z) {
      return gemm_nn<T>(st, n, n, n, 1.0, X, n, Y, n, beta, Z, n);
    };

    // X = 2^-s A^H, D = 2^-s G
    const double f = std::ldexp(1.0, -plan.s);
    CLM_CUDA(launch_transpose<T>(st, n, n, f, A, lda, ws.Xs, n, true));
    CLM_CUDA(launch_scale_copy<T>(st, n, f, G, ldg, ws.Ds, n));

    // even powers and their derivatives (the forward pass's order: A4 = A2 A2,
    // A6 = A4 A2, A8 = A4 A4)
    T **P = ws.P, **M = ws.M;
    CLM_CUDA(mm(ws.Xs, ws.Xs, 0.0, P[0]));
    CLM_CUDA(mm(ws.Xs, ws.Ds, 0.0, M[0]));
    CLM_CUDA(mm(ws.Ds, ws.Xs, 1.0, M[0]));
    if (np >= 2) {
      CLM_CUDA(mm(P[0], P[0], 0.0, P[1]));
      CLM_CUDA(mm(P[0], M[0], 0.0, M[1]));
      CLM_CUDA(mm(M[0], P[0], 1.0, M[1]));
    }
    if (np >= 3) {
      CLM_CUDA(mm(P[1], P[0], 0.0, P[2]));
      CLM_CUDA(mm(M[1], P[0], 0.0, M[2]));
      CLM_CUDA(mm(P[1], M[0], 1.0, M[2]));
    }
    if (np >= 4) {
      CLM_CUDA(mm(P[1], P[1], 0.0, P[3]));
      CLM_CUDA(mm(P[1], M[1], 0.0, M[3]));
      CLM_CUDA(mm(M[1], P[1], 1.0, M[3]));
    }

    if (m != 13) {
      double cv[5] = {0, 0, 0, 0, 0}, cw[5] = {0, 0, 0, 0, 0};
      for (int i = 0; i <= np; ++i) {
        cv[i] = b[2 * i];
        cw[i] = b[2 * i + 1];
      }
      CLM_CUDA(launch_pade_even_odd<T>(st, n, np, P[0], P[1], P[2], P[3], cv, cw, ws.V, ws.W));
      cv[0] = 0.0;
      cw[0] = 0.0;  // the derivative of the identity term is zero
      CLM_CUDA(launch_pade_even_odd<T>(st, n, np, M[0], M[1], M[2], M[3], cv, cw, ws.LV, ws.LW));
    } else {
      // odd: W1 = b9 A2 + b11 A4 + b13 A6, W = b1 I + b3 A2 + b5 A4 + b7 A6 + A6 W1
      const double co[5] = {0.0, b[9], b[11], b[13], 0.0};
      const double cwo[5] = {b[1], b[3], b[5], b[7], 0.0};
      const double cwo0[5] = {0.0, b[3], b[5], b[7], 0.0};
      CLM_CUDA(launch_pade_even_odd<T>(st, n, 3, P[0], P[1], P[2], nullptr, co, cwo, ws.T1, ws.W));
      CLM_CUDA(launch_pade_even_odd<T>(st, n, 3, M[0], M[1], M[2], nullptr, co, cwo0, ws.T2, ws.LW));
      CLM_CUDA(mm(P[2], ws.T2, 1.0, ws.LW));  // dW += A6 dW1 + dA6 W1
      CLM_CUDA(mm(M[2], ws.T1, 1.0, ws.LW));
      CLM_CUDA(mm(P[2], ws.T1, 1.0, ws.W));
      // even: Z1 = b8 A2 + b10 A4 + b12 A6, V = b0 I + b2 A2 + b4 A4 + b6 A6 + A6 Z1
      const double ce[5] = {0.0, b[8], b[10], b[12], 0.0};
      const double cve[5] = {b[0], b[2], b[4], b[6], 0.0};
      const double cve0[5] = {0.0, b[2], b[4], b[6], 0.0};
      CLM_CUDA(launch_pade_even_odd<T>(st, n, 3, P[0], P[1], P[2], nullptr, ce, cve, ws.T1, ws.V));
      CLM_CUDA(launch_pade_even_odd<T>(st, n, 3, M[0], M[1], M[2], nullptr, ce, cve0, ws.T2, ws.LV));
      CLM_CUDA(mm(P[2], ws.T2, 1.0, ws.LV));
      CLM_CUDA(mm(M[2], ws.T1, 1.0, ws.LV));
      CLM_CUDA(mm(P[2], ws.T1, 1.0, ws.V));
    }
    // U = X W, dU = X dW + D W
    CLM_CUDA(mm(ws.Xs, ws.W, 0.0, ws.T1));
    CLM_CUDA(mm(ws.Xs, ws.LW, 0.0, ws.T2));
    CLM_CUDA(mm(ws.Ds, ws.W, 1.0, ws.T2));
    // p = V + U over T1, q = V - U over V; dp over T2, dq over LV
    CLM_CUDA(launch_pade_split<T>(st, n, ws.T1, ws.V, ws.T1, n, ws.V));
    CLM_CUDA(launch_pade_split<T>(st, n, ws.T2, ws.LV, ws.T2, n, ws.LV));
    // R = q^-1 p; dR = q^-1 (dp - dq R)
    T *Rm = P[0], *Lm = M[0];
    CLM_CUDA(getrf<T>(st, n, ws.V, n, ws.lu, d_info));
    CLM_CUDA(getrs<T>(st, n, n, ws.V, n, ws.lu, ws.T1, n, Rm, n, d_info + 1));
    CLM_CUDA(gemm_nn<T>(st, n, n, n, -1.0, ws.LV, n, Rm, n, 1.0, ws.T2, n));
    CLM_CUDA(getrs<T>(st, n, n, ws.V, n, ws.lu, ws.T2, n, Lm, n, d_info + 1));

    if (elem<T>::single && plan.s > 0) {
      // single tiers square in FP64, like expm
      using Wd = typename Wide<T>::type;
      const std::size_t nn = (std::size_t)n * n;
      Wd *r = ws.wide, *l = ws.wide + nn, *r2 = ws.wide + 2 * nn, *l2 = ws.wide + 3 * nn;
      CLM_CUDA((launch_convert<T, Wd>(st, n, Rm, n, r, n)));
      CLM_CUDA((launch_convert<T, Wd>(st, n, Lm, n, l, n)));
      CLM_CUDA(frechet_squarings<Wd>(st, n, plan.s, &r, &l, &r2, &l2));
      CLM_CUDA((launch_convert<Wd, T>(st, n, l, n, gradA, ldga)));
      if (E) {
        CLM_CUDA((launch_convert<Wd, T>(st, n, r, n, ws.T1, n)));
        CLM_CUDA(launch_transpose<T>(st, n, n, 1.0, ws.T1, n, E, lde, true));
      }
      return ok_status();
    }
    T *r2 = ws.T1, *l2 = ws.LW;
    CLM_CUDA(frechet_squarings<T>(st, n, plan.s, &Rm, &Lm, &r2, &l2));
    CLM_CUDA(launch_scale_copy<T>(st, n, 1.0, Lm, n, gradA, ldga));
    // g(A^H) = g(A)^H
    if (E) CLM_CUDA(launch_transpose<T>(st, n, n, 1.0, Rm, n, E, lde, true));
    return ok_status();
  };
  if (blas == nullptr) return post();
  CallKey key;
  key.mix((unsigned long long)n | ((unsigned long long)plan.m << 32) | ((unsigned long long)plan.s << 48));
  key.mix(A);
  key.mix(G);
  key.mix(gradA);
  key.mix(E);
  key.mix((unsigned long long)lda | ((unsigned long long)ldg << 32));
  key.mix((unsigned long long)ldga | ((unsigned long long)lde << 32));
  key.mix(work);
  key.mix((unsigned long long)lwork);
  key.mix(d_info);
  key.mix(st);
  key.mix((unsigned long long)blas->split_terms | ((unsigned long long)(blas->fp64_digits + 16) << 32));
  key.mix(blas->work);
  key.mix((unsigned long long)blas->work_bytes);
  return run_or_replay(&blas->expm_graphs, blas->vjp[type_slot<T>()], st, key.h, post);
}

}  // namespace
}  // namespace clm

using namespace clm;

extern "C" {

#define CLM_VJP_API(SUF, T, PT, CPT)                                                               \
  calamanStatus_t calaman_expm_vjp_bufferSize_##SUF(calamanSolverHandle_t h, int n, size_t *bytes) { \
    if (n < 1 || n > kMaxDim || bytes == nullptr) return blas_status(CALAMAN_STATUS_INVALID_VALUE); \
    *bytes = vjp_bytes<T>(h, n);                                                                   \
    return ok_status();                                                                            \
  }                                                                                                \
  calamanStatus_t calaman_expm_vjp_##SUF(calamanBlasHandle_t blas, calamanSolverHandle_t,          \
                                         calamanStream_t stream, int n, CPT A, int lda, CPT G,     \
                                         int ldg, PT gradA, int ldga, PT E, int lde, void *work,   \
                                         size_t lwork, int *d_info, calamanExpmPlan_t *plan) {     \
    return vjp_api<T>(blas, stream, n, reinterpret_cast<const T *>(A), lda,                       \
                      reinterpret_cast<const T *>(G), ldg, reinterpret_cast<T *>(gradA), ldga,     \
                      reinterpret_cast<T *>(E), lde, work, lwork, d_info, plan);                   \
  }
CLM_VJP_API(s, float, float *, const float *)
CLM_VJP_API(d, double, double *, const double *)
CLM_VJP_API(c, float2, void *, const void *)
CLM_VJP_API(z, double2, void *, const void *)
#undef CLM_VJP_API

}  // extern "C"
