// calaman_b200.hpp -- C++ drop-in for calaman_G's `calaman.expm`,
// `calaman.paterson_stockmeyer` and `calaman.horner` module interfaces.
//
// A reference call site such as
//
//     import calaman.expm;
//     calaman::Status st = calaman::expm<double>(blas, solver, stream, n, d_A, lda,
//                                                d_E, lde, d_work, bytes, d_info, &plan);
//
// compiles unchanged against this header once `blas` / `solver` are
// calaman::BlasHandle / calaman::SolverHandle (both a calamanHandle_t) and the
// stream is a cudaStream_t. The templates forward to the C ABI in
// calaman_b200.h; Status keeps the reference's {domain, code} shape, its ok(),
// name() and outcome equality (src/error_handling/error_handling.cppm:99-187).
// Element types: float, double, std::complex<float>, std::complex<double>
// (interleaved, layout-compatible with the reference's wwrFloatComplex /
// wwrDoubleComplex); horner and paterson_stockmeyer exist for float and double.
#pragma once

#include <array>
#include <complex>
#include <cstddef>
#include <type_traits>

#include "calaman_b200.h"

// cudaStream_t exactly as the CUDA runtime declares it, so this header also
// compiles in translation units that include no CUDA header.
struct CUstream_st;
typedef struct CUstream_st *cudaStream_t;

namespace calaman {

enum class ErrorDomain { blas = CALAMAN_DOMAIN_BLAS, solver = CALAMAN_DOMAIN_SOLVER, runtime = CALAMAN_DOMAIN_RUNTIME };

struct Status {
  ErrorDomain domain = ErrorDomain::blas;
  int code = 0;
  constexpr Status() = default;
  constexpr Status(calamanStatus_t s) : domain(static_cast<ErrorDomain>(s.domain)), code(s.code) {}
  [[nodiscard]] constexpr bool ok() const noexcept { return code == 0; }
  [[nodiscard]] const char *name() const noexcept {
    if (domain == ErrorDomain::runtime) return ok() ? "cudaSuccess" : "cudaError";
    switch (code) {
    case CALAMAN_STATUS_SUCCESS: return "SUCCESS";
    case CALAMAN_STATUS_NOT_INITIALIZED: return "NOT_INITIALIZED";
    case CALAMAN_STATUS_ALLOC_FAILED: return "ALLOC_FAILED";
    case CALAMAN_STATUS_INVALID_VALUE: return "INVALID_VALUE";
    case CALAMAN_STATUS_ARCH_MISMATCH: return "ARCH_MISMATCH";
    case CALAMAN_STATUS_EXECUTION_FAILED: return "EXECUTION_FAILED";
    case CALAMAN_STATUS_INTERNAL_ERROR: return "INTERNAL_ERROR";
    case CALAMAN_STATUS_NOT_SUPPORTED: return "NOT_SUPPORTED";
    default: return "UNKNOWN";
    }
  }
  // every success equals every other success; errors compare by domain and code
  [[nodiscard]] constexpr bool operator==(const Status &o) const noexcept {
    if (ok() || o.ok()) return ok() && o.ok();
    return domain == o.domain && code == o.code;
  }
};

using BlasHandle = calamanHandle_t;
using SolverHandle = calamanHandle_t;
using ExpmPlan = calamanExpmPlan_t;
using PatersonStockmeyerPlan = calamanPatersonStockmeyerPlan_t;

template <typename T>
using real_t = std::conditional_t<std::is_same_v<T, std::complex<float>>, float,
                                  std::conditional_t<std::is_same_v<T, std::complex<double>>, double, T>>;

namespace detail {
template <typename T> inline constexpr bool is_single = std::is_same_v<real_t<T>, float>;
template <typename T> inline constexpr bool is_complex =
    std::is_same_v<T, std::complex<float>> || std::is_same_v<T, std::complex<double>>;
template <typename T> struct always_false : std::false_type {};
}  // namespace detail

// ---- plan (src/expm/plan.cppm:51-130) ---------------------------------------
template <typename T> real_t<T> pade_theta(int m) {
  if constexpr (detail::is_single<T>) return calaman_pade_theta_s(m);
  else return calaman_pade_theta_d(m);
}
template <typename T> ExpmPlan expm_plan(real_t<T> norm1) {
  if constexpr (detail::is_single<T>) return calaman_expm_plan_s(norm1);
  else return calaman_expm_plan_d(norm1);
}

// ---- workspace queries (src/expm/buffer_size.cppm) ----------------------------
template <typename T> Status expm_bufferSize(SolverHandle h, int n, std::size_t *bytes) {
  if constexpr (std::is_same_v<T, float>) return calaman_expm_bufferSize_s(h, n, bytes);
  else if constexpr (std::is_same_v<T, double>) return calaman_expm_bufferSize_d(h, n, bytes);
  else if constexpr (std::is_same_v<T, std::complex<float>>) return calaman_expm_bufferSize_c(h, n, bytes);
  else return calaman_expm_bufferSize_z(h, n, bytes);
}
template <typename T> Status pade_bufferSize(SolverHandle h, int m, int n, std::size_t *bytes) {
  if constexpr (std::is_same_v<T, float>) return calaman_pade_bufferSize_s(h, m, n, bytes);
  else if constexpr (std::is_same_v<T, double>) return calaman_pade_bufferSize_d(h, m, n, bytes);
  else if constexpr (std::is_same_v<T, std::complex<float>>) return calaman_pade_bufferSize_c(h, m, n, bytes);
  else return calaman_pade_bufferSize_z(h, m, n, bytes);
}

// ---- expm (src/expm/expm.cppm:87-174) ------------------------------------------
template <typename T>
Status expm(BlasHandle blas, SolverHandle solver, cudaStream_t stream, int n, const T *d_A, int lda,
            T *d_expA, int lde, void *d_work, std::size_t lwork_bytes, int *d_info,
            ExpmPlan *plan = nullptr) {
  if constexpr (std::is_same_v<T, float>)
    return calaman_expm_s(blas, solver, stream, n, d_A, lda, d_expA, lde, d_work, lwork_bytes, d_info, plan);
  else if constexpr (std::is_same_v<T, double>)
    return calaman_expm_d(blas, solver, stream, n, d_A, lda, d_expA, lde, d_work, lwork_bytes, d_info, plan);
  else if constexpr (std::is_same_v<T, std::complex<float>>)
    return calaman_expm_c(blas, solver, stream, n, d_A, lda, d_expA, lde, d_work, lwork_bytes, d_info, plan);
  else
    return calaman_expm_z(blas, solver, stream, n, d_A, lda, d_expA, lde, d_work, lwork_bytes, d_info, plan);
}

// ---- expm_vjp: the adjoint of expm (new entry, no reference counterpart) -------
template <typename T> Status expm_vjp_bufferSize(SolverHandle h, int n, std::size_t *bytes) {
  if constexpr (std::is_same_v<T, float>) return calaman_expm_vjp_bufferSize_s(h, n, bytes);
  else if constexpr (std::is_same_v<T, double>) return calaman_expm_vjp_bufferSize_d(h, n, bytes);
  else if constexpr (std::is_same_v<T, std::complex<float>>) return calaman_expm_vjp_bufferSize_c(h, n, bytes);
  else return calaman_expm_vjp_bufferSize_z(h, n, bytes);
}
// d_gradA = L(A^H, G); d_expA may be nullptr
template <typename T>
Status expm_vjp(BlasHandle blas, SolverHandle solver, cudaStream_t stream, int n, const T *d_A, int lda,
                const T *d_G, int ldg, T *d_gradA, int ldga, T *d_expA, int lde, void *d_work,
                std::size_t lwork_bytes, int *d_info, ExpmPlan *plan = nullptr) {
  if constexpr (std::is_same_v<T, float>)
    return calaman_expm_vjp_s(blas, solver, stream, n, d_A, lda, d_G, ldg, d_gradA, ldga, d_expA, lde, d_work,
                              lwork_bytes, d_info, plan);
  else if constexpr (std::is_same_v<T, double>)
    return calaman_expm_vjp_d(blas, solver, stream, n, d_A, lda, d_G, ldg, d_gradA, ldga, d_expA, lde, d_work,
                              lwork_bytes, d_info, plan);
  else if constexpr (std::is_same_v<T, std::complex<float>>)
    return calaman_expm_vjp_c(blas, solver, stream, n, d_A, lda, d_G, ldg, d_gradA, ldga, d_expA, lde, d_work,
                              lwork_bytes, d_info, plan);
  else
    return calaman_expm_vjp_z(blas, solver, stream, n, d_A, lda, d_G, ldg, d_gradA, ldga, d_expA, lde, d_work,
                              lwork_bytes, d_info, plan);
}

// ---- expm_batched / expm_vjp_batched (new entries): float and double ----------
template <typename T> Status expm_batched_bufferSize(SolverHandle h, int batch, const int *h_n, std::size_t *bytes) {
  static_assert(std::is_same_v<T, float> || std::is_same_v<T, double>, "expm_batched: float or double");
  if constexpr (std::is_same_v<T, float>) return calaman_expm_batched_bufferSize_s(h, batch, h_n, bytes);
  else return calaman_expm_batched_bufferSize_d(h, batch, h_n, bytes);
}
template <typename T>
Status expm_batched(BlasHandle blas, SolverHandle solver, cudaStream_t stream, int batch, const int *h_n,
                    const T *const *h_A, const int *h_lda, T *const *h_expA, const int *h_lde, void *d_work,
                    std::size_t lwork_bytes, int *d_info, ExpmPlan *h_plans = nullptr) {
  static_assert(std::is_same_v<T, float> || std::is_same_v<T, double>, "expm_batched: float or double");
  if constexpr (std::is_same_v<T, float>)
    return calaman_expm_batched_s(blas, solver, stream, batch, h_n, h_A, h_lda, h_expA, h_lde, d_work,
                                  lwork_bytes, d_info, h_plans);
  else
    return calaman_expm_batched_d(blas, solver, stream, batch, h_n, h_A, h_lda, h_expA, h_lde, d_work,
                                  lwork_bytes, d_info, h_plans);
}
template <typename T>
Status expm_vjp_batched_bufferSize(SolverHandle h, int batch, const int *h_n, std::size_t *bytes) {
  static_assert(std::is_same_v<T, float> || std::is_same_v<T, double>, "expm_vjp_batched: float or double");
  if constexpr (std::is_same_v<T, float>) return calaman_expm_vjp_batched_bufferSize_s(h, batch, h_n, bytes);
  else return calaman_expm_vjp_batched_bufferSize_d(h, batch, h_n, bytes);
}
template <typename T>
Status expm_vjp_batched(BlasHandle blas, SolverHandle solver, cudaStream_t stream, int batch, const int *h_n,
                        const T *const *h_A, const int *h_lda, const T *const *h_G, const int *h_ldg,
                        T *const *h_gradA, const int *h_ldga, T *const *h_expA, const int *h_lde, void *d_work,
                        std::size_t lwork_bytes, int *d_info, ExpmPlan *h_plans = nullptr) {
  static_assert(std::is_same_v<T, float> || std::is_same_v<T, double>, "expm_vjp_batched: float or double");
  if constexpr (std::is_same_v<T, float>)
    return calaman_expm_vjp_batched_s(blas, solver, stream, batch, h_n, h_A, h_lda, h_G, h_ldg, h_gradA, h_ldga,
                                      h_expA, h_lde, d_work, lwork_bytes, d_info, h_plans);
  else
    return calaman_expm_vjp_batched_d(blas, solver, stream, batch, h_n, h_A, h_lda, h_G, h_ldg, h_gradA, h_ldga,
                                      h_expA, h_lde, d_work, lwork_bytes, d_info, h_plans);
}

// ---- gebal, scaling job (src/lapack/gebal/interface.cppm:100-255) ---------------
enum class GebalJob { None = 0, Permute = 1, Scale = 2, Both = 3 };
inline constexpr int gebal_default_max_sweeps = 1000;
template <typename T> Status gebal_bufferSize(int n, int *lwork_ints) {
  return calaman_gebal_bufferSize(n, lwork_ints);
}
template <typename T>
Status gebal(cudaStream_t stream, GebalJob job, int n, T *d_A, int lda, int *ilo, int *ihi, real_t<T> *d_scale,
             int *d_work, int max_sweeps = gebal_default_max_sweeps) {
  const int j = static_cast<int>(job);
  if constexpr (std::is_same_v<T, float>)
    return calaman_gebal_s(stream, j, n, d_A, lda, ilo, ihi, d_scale, d_work, max_sweeps, nullptr);
  else if constexpr (std::is_same_v<T, double>)
    return calaman_gebal_d(stream, j, n, d_A, lda, ilo, ihi, d_scale, d_work, max_sweeps, nullptr);
  else if constexpr (std::is_same_v<T, std::complex<float>>)
    return calaman_gebal_c(stream, j, n, d_A, lda, ilo, ihi, d_scale, d_work, max_sweeps, nullptr);
  else
    return calaman_gebal_z(stream, j, n, d_A, lda, ilo, ihi, d_scale, d_work, max_sweeps, nullptr);
}

// ---- expm_herm (src/expm/expm_herm.cppm:70-199) and its eigensolver ---------------
enum class FillMode : int { Lower = CALAMAN_FILL_MODE_LOWER, Upper = CALAMAN_FILL_MODE_UPPER };
template <typename T> Status expm_herm_bufferSize(SolverHandle h, FillMode uplo, int n, std::size_t *bytes) {
  const int u = static_cast<int>(uplo);
  if constexpr (std::is_same_v<T, float>) return calaman_expm_herm_bufferSize_s(h, u, n, bytes);
  else if constexpr (std::is_same_v<T, double>) return calaman_expm_herm_bufferSize_d(h, u, n, bytes);
  else if constexpr (std::is_same_v<T, std::complex<float>>) return calaman_expm_herm_bufferSize_c(h, u, n, bytes);
  else return calaman_expm_herm_bufferSize_z(h, u, n, bytes);
}
template <typename T>
Status expm_herm(BlasHandle blas, SolverHandle solver, cudaStream_t stream, FillMode uplo, int n, const T *d_A,
                 int lda, T *d_expA, int lde, void *d_work, std::size_t lwork_bytes, int *d_info) {
  const int u = static_cast<int>(uplo);
  if constexpr (std::is_same_v<T, float>)
    return calaman_expm_herm_s(blas, solver, stream, u, n, d_A, lda, d_expA, lde, d_work, lwork_bytes, d_info);
  else if constexpr (std::is_same_v<T, double>)
    return calaman_expm_herm_d(blas, solver, stream, u, n, d_A, lda, d_expA, lde, d_work, lwork_bytes, d_info);
  else if constexpr (std::is_same_v<T, std::complex<float>>)
    return calaman_expm_herm_c(blas, solver, stream, u, n, d_A, lda, d_expA, lde, d_work, lwork_bytes, d_info);
  else
    return calaman_expm_herm_z(blas, solver, stream, u, n, d_A, lda, d_expA, lde, d_work, lwork_bytes, d_info);
}
template <typename T> Status heevd_bufferSize(FillMode uplo, int n, std::size_t *bytes) {
  const int u = static_cast<int>(uplo);
  if constexpr (std::is_same_v<T, float>) return calaman_heevd_bufferSize_s(u, n, bytes);
  else if constexpr (std::is_same_v<T, double>) return calaman_heevd_bufferSize_d(u, n, bytes);
  else if constexpr (std::is_same_v<T, std::complex<float>>) return calaman_heevd_bufferSize_c(u, n, bytes);
  else return calaman_heevd_bufferSize_z(u, n, bytes);
}
template <typename T>
Status heevd(cudaStream_t stream, FillMode uplo, int n, T *d_A, int lda, real_t<T> *d_w, void *d_work,
             std::size_t lwork_bytes, int *d_info) {
  const int u = static_cast<int>(uplo);
  if constexpr (std::is_same_v<T, float>)
    return calaman_heevd_s(stream, u, n, d_A, lda, d_w, d_work, lwork_bytes, d_info);
  else if constexpr (std::is_same_v<T, double>)
    return calaman_heevd_d(stream, u, n, d_A, lda, d_w, d_work, lwork_bytes, d_info);
  else if constexpr (std::is_same_v<T, std::complex<float>>)
    return calaman_heevd_c(stream, u, n, d_A, lda, d_w, d_work, lwork_bytes, d_info);
  else
    return calaman_heevd_z(stream, u, n, d_A, lda, d_w, d_work, lwork_bytes, d_info);
}

// ---- geodesic trial points (src/cg_unitary/geodesic_search.cppm:338-420) ----------
template <typename T> Status geodesic_points_bufferSize(SolverHandle h, int n, int num_samples, std::size_t *bytes) {
  if constexpr (std::is_same_v<T, float>) return calaman_geodesic_points_bufferSize_s(h, n, num_samples, bytes);
  else if constexpr (std::is_same_v<T, double>) return calaman_geodesic_points_bufferSize_d(h, n, num_samples, bytes);
  else if constexpr (std::is_same_v<T, std::complex<float>>)
    return calaman_geodesic_points_bufferSize_c(h, n, num_samples, bytes);
  else return calaman_geodesic_points_bufferSize_z(h, n, num_samples, bytes);
}
template <typename T>
Status geodesic_points(BlasHandle blas, SolverHandle solver, cudaStream_t stream, int n, const T *d_W, int ldw,
                       const T *d_H, int ldh, real_t<T> step, int num_samples, T *d_Wout, void *d_work,
                       std::size_t lwork_bytes, int *d_info) {
  const double mu = static_cast<double>(step);
  if constexpr (std::is_same_v<T, float>)
    return calaman_geodesic_points_s(blas, solver, stream, n, d_W, ldw, d_H, ldh, mu, num_samples, d_Wout, d_work,
                                     lwork_bytes, d_info);
  else if constexpr (std::is_same_v<T, double>)
    return calaman_geodesic_points_d(blas, solver, stream, n, d_W, ldw, d_H, ldh, mu, num_samples, d_Wout, d_work,
                                     lwork_bytes, d_info);
  else if constexpr (std::is_same_v<T, std::complex<float>>)
    return calaman_geodesic_points_c(blas, solver, stream, n, d_W, ldw, d_H, ldh, mu, num_samples, d_Wout, d_work,
                                     lwork_bytes, d_info);
  else
    return calaman_geodesic_points_z(blas, solver, stream, n, d_W, ldw, d_H, ldh, mu, num_samples, d_Wout, d_work,
                                     lwork_bytes, d_info);
}

// ---- lacn2 (src/lapack/lacn2/interface.cppm:85-200) -------------------------------
template <typename T> std::size_t lacn2_bufferSize(int n) {
  static_assert(std::is_same_v<T, float> || std::is_same_v<T, double>, "lacn2 is real only");
  if constexpr (std::is_same_v<T, float>) return calaman_lacn2_bufferSize_s(n);
  else return calaman_lacn2_bufferSize_d(n);
}
template <typename T>
Status lacn2(BlasHandle handle, int n, T *d_v, T *d_x, void *d_work, std::size_t work_bytes, T &est,
             int &kase, std::array<int, 3> &isave) {
  static_assert(std::is_same_v<T, float> || std::is_same_v<T, double>, "lacn2 is real only");
  if constexpr (std::is_same_v<T, float>)
    return calaman_lacn2_s(handle, n, d_v, d_x, d_work, work_bytes, &est, &kase, isave.data());
  else
    return calaman_lacn2_d(handle, n, d_v, d_x, d_work, work_bytes, &est, &kase, isave.data());
}

// ---- expm_balanced: D exp(D^-1 A D) D^-1 (new entry) ----------------------------
template <typename T> Status expm_balanced_bufferSize(SolverHandle h, int n, std::size_t *bytes) {
  if constexpr (std::is_same_v<T, float>) return calaman_expm_balanced_bufferSize_s(h, n, bytes);
  else if constexpr (std::is_same_v<T, double>) return calaman_expm_balanced_bufferSize_d(h, n, bytes);
  else if constexpr (std::is_same_v<T, std::complex<float>>) return calaman_expm_balanced_bufferSize_c(h, n, bytes);
  else return calaman_expm_balanced_bufferSize_z(h, n, bytes);
}
template <typename T>
Status expm_balanced(BlasHandle blas, SolverHandle solver, cudaStream_t stream, int n, const T *d_A, int lda,
                     T *d_expA, int lde, void *d_work, std::size_t lwork_bytes, int *d_info,
                     ExpmPlan *plan = nullptr) {
  if constexpr (std::is_same_v<T, float>)
    return calaman_expm_balanced_s(blas, solver, stream, n, d_A, lda, d_expA, lde, d_work, lwork_bytes, d_info, plan);
  else if constexpr (std::is_same_v<T, double>)
    return calaman_expm_balanced_d(blas, solver, stream, n, d_A, lda, d_expA, lde, d_work, lwork_bytes, d_info, plan);
  else if constexpr (std::is_same_v<T, std::complex<float>>)
    return calaman_expm_balanced_c(blas, solver, stream, n, d_A, lda, d_expA, lde, d_work, lwork_bytes, d_info, plan);
  else
    return calaman_expm_balanced_z(blas, solver, stream, n, d_A, lda, d_expA, lde, d_work, lwork_bytes, d_info, plan);
}

// ---- pade (src/expm/pade.cppm:77-191) ------------------------------------------
template <typename T>
Status pade(BlasHandle blas, SolverHandle solver, cudaStream_t stream, int m, int n, const T *d_A,
            int lda, T *d_r, int ldr, void *d_work, std::size_t lwork_bytes, int *d_info) {
  if constexpr (std::is_same_v<T, float>)
    return calaman_pade_s(blas, solver, stream, m, n, d_A, lda, d_r, ldr, d_work, lwork_bytes, d_info);
  else if constexpr (std::is_same_v<T, double>)
    return calaman_pade_d(blas, solver, stream, m, n, d_A, lda, d_r, ldr, d_work, lwork_bytes, d_info);
  else if constexpr (std::is_same_v<T, std::complex<float>>)
    return calaman_pade_c(blas, solver, stream, m, n, d_A, lda, d_r, ldr, d_work, lwork_bytes, d_info);
  else
    return calaman_pade_z(blas, solver, stream, m, n, d_A, lda, d_r, ldr, d_work, lwork_bytes, d_info);
}

// ---- matrix_norm1 (src/expm/norm1.cppm:45-56) -------------------------------------
template <typename T>
real_t<T> matrix_norm1(cudaStream_t stream, int n, const T *d_A, int lda, real_t<T> *d_colsum) {
  if constexpr (std::is_same_v<T, float>) return calaman_matrix_norm1_s(stream, n, d_A, lda, d_colsum);
  else if constexpr (std::is_same_v<T, double>) return calaman_matrix_norm1_d(stream, n, d_A, lda, d_colsum);
  else if constexpr (std::is_same_v<T, std::complex<float>>) return calaman_matrix_norm1_c(stream, n, d_A, lda, d_colsum);
  else return calaman_matrix_norm1_z(stream, n, d_A, lda, d_colsum);
}

// ---- horner (src/horner/interface.cppm:104-194) --------------------------------
template <typename T> std::size_t horner_bufferSize(int n) {
  static_assert(std::is_same_v<T, float> || std::is_same_v<T, double>, "horner: float or double");
  if constexpr (std::is_same_v<T, float>) return calaman_horner_bufferSize_s(n);
  else return calaman_horner_bufferSize_d(n);
}
template <typename T>
Status horner(BlasHandle handle, int n, const T *d_coeffs, int degree, const T *d_A, int lda, T *d_P,
              int ldp, void *d_work, std::size_t work_bytes) {
  static_assert(std::is_same_v<T, float> || std::is_same_v<T, double>, "horner: float or double");
  if constexpr (std::is_same_v<T, float>)
    return calaman_horner_s(handle, n, d_coeffs, degree, d_A, lda, d_P, ldp, d_work, work_bytes);
  else
    return calaman_horner_d(handle, n, d_coeffs, degree, d_A, lda, d_P, ldp, d_work, work_bytes);
}

// ---- paterson_stockmeyer (src/paterson_stockmeyer/interface.cppm:117-422) --------
inline int paterson_stockmeyer_cost(int degree, int s) { return calaman_paterson_stockmeyer_cost(degree, s); }
inline int paterson_stockmeyer_block_size(int degree) { return calaman_paterson_stockmeyer_block_size(degree); }
inline PatersonStockmeyerPlan paterson_stockmeyer_plan(int degree, int s_requested = 0) {
  return calaman_paterson_stockmeyer_plan(degree, s_requested);
}
template <typename T> std::size_t paterson_stockmeyer_power_stride(int n) {
  if constexpr (std::is_same_v<T, float>) return calaman_paterson_stockmeyer_power_stride_s(n);
  else return calaman_paterson_stockmeyer_power_stride_d(n);
}
template <typename T>
std::size_t paterson_stockmeyer_bufferSize(int n, int degree, int s_requested = 0) {
  if constexpr (std::is_same_v<T, float>) return calaman_paterson_stockmeyer_bufferSize_s(n, degree, s_requested);
  else return calaman_paterson_stockmeyer_bufferSize_d(n, degree, s_requested);
}
template <typename T>
Status paterson_stockmeyer(BlasHandle handle, int n, const T *d_coeffs, int degree, const T *d_A,
                           int lda, T *d_P, int ldp, void *d_work, std::size_t work_bytes,
                           int s_requested = 0) {
  static_assert(std::is_same_v<T, float> || std::is_same_v<T, double>,
                "paterson_stockmeyer: float or double");
  if constexpr (std::is_same_v<T, float>)
    return calaman_paterson_stockmeyer_s(handle, n, d_coeffs, degree, d_A, lda, d_P, ldp, d_work,
                                         work_bytes, s_requested);
  else
    return calaman_paterson_stockmeyer_d(handle, n, d_coeffs, degree, d_A, lda, d_P, ldp, d_work,
                                         work_bytes, s_requested);
}

}  // namespace calaman
