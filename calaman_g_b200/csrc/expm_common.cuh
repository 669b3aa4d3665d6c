// expm_common.cuh -- the Pade tables, the (m, s) plan and small host helpers
// shared by the expm / pade drivers, the adjoint (VJP) driver and the batched
// driver.
#pragma once

#include <cmath>
#include <type_traits>

#include "kernels.cuh"

namespace clm {

inline KernelTimer *timer_of(calamanHandle_t h) { return h ? &h->timer : nullptr; }
inline int split_terms_of(calamanHandle_t h) { return h ? h->split_terms : 6; }

inline constexpr int kMaxDim = 46340;  // flat int indexing bound, src/expm/detail.cppm:25-28

// ---- Pade tables (src/expm/expm_bridge.h:58-91; Higham 2005 eq. 2.2) -------
inline constexpr double kB3[4] = {1.0, 1.0 / 2.0, 1.0 / 10.0, 1.0 / 120.0};
inline constexpr double kB5[6] = {1.0, 1.0 / 2.0, 1.0 / 9.0, 1.0 / 72.0, 1.0 / 1008.0, 1.0 / 30240.0};
inline constexpr double kB7[8] = {1.0,          1.0 / 2.0,     3.0 / 26.0,     5.0 / 312.0,
                           5.0 / 3432.0, 1.0 / 11440.0, 1.0 / 308880.0, 1.0 / 17297280.0};
inline constexpr double kB9[10] = {1.0,            1.0 / 2.0,        2.0 / 17.0,       7.0 / 408.0,
                            7.0 / 4080.0,   1.0 / 8160.0,     1.0 / 159120.0,   1.0 / 4455360.0,
                            1.0 / 196035840.0, 1.0 / 17643225600.0};
inline constexpr double kB13[14] = {1.0,
                             1.0 / 2.0,
                             3.0 / 25.0,
                             11.0 / 600.0,
                             11.0 / 5520.0,
                             3.0 / 18400.0,
                             1.0 / 96600.0,
                             1.0 / 1932000.0,
                             1.0 / 48944000.0,
                             1.0 / 1585785600.0,
                             1.0 / 67395888000.0,
                             1.0 / 3953892096000.0,
                             1.0 / 355850288640000.0,
                             1.0 / 64764752532480000.0};

inline const double *pade_coeffs(int m) {
  switch (m) {
  case 3: return kB3;
  case 5: return kB5;
  case 7: return kB7;
  case 9: return kB9;
  case 13: return kB13;
  default: return nullptr;
  }
}
inline int pade_num_powers(int m) { return (m == 13) ? 3 : (m - 1) / 2; }
inline int pade_num_gemms(int m) { return pade_num_powers(m) + 1 + ((m == 13) ? 2 : 0); }

// theta_m, src/expm/plan.cppm:51-85: u = 2^-53 and u = 2^-24 columns.
inline double theta_double(int m) {
  switch (m) {
  case 3: return 1.495585217958292e-2;
  case 5: return 2.539398330063232e-1;
  case 7: return 9.504178996162932e-1;
  case 9: return 2.097847961257067;
  case 13: return 5.371920351148152;
  default: return 0.0;
  }
}
inline float theta_single(int m) {
  switch (m) {
  case 3: return 4.258730034897931e-1f;
  case 5: return 1.880152698533769f;
  case 7: return 3.925724846433284f;
  case 9: return 6.249156334514102f;
  case 13: return 1.124873763647540e1f;
  default: return 0.0f;
  }
}

// expm_plan<T>, src/expm/plan.cppm:112-130 (the single column is compared and
// log2'd in float, as the reference's float instantiation does).
template <typename R>
inline calamanExpmPlan_t plan_for(R norm1) {
  static const int degrees[5] = {3, 5, 7, 9, 13};
  for (int m : degrees) {
    const R th = sizeof(R) == 4 ? (R)theta_single(m) : (R)theta_double(m);
    if (norm1 <= th) return calamanExpmPlan_t{m, 0, pade_num_gemms(m)};
  }
  const R theta = sizeof(R) == 4 ? (R)theta_single(13) : (R)theta_double(13);
  int s = (int)std::ceil(std::log2(norm1 / theta));
  if (s < 0) s = 0;
  return calamanExpmPlan_t{13, s, pade_num_gemms(13) + s};
}

// FP32 and complex64 products run as split-BF16 tensor-core GEMMs and need
// operand-part scratch sized for the largest (n x n x n) product of the
// evaluation.
template <typename T> inline std::size_t tc_scratch_bytes(int n) {
  if (std::is_same<T, float>::value) return tc_gemm_workspace_bytes(n, n, n, 6);
  if (std::is_same<T, float2>::value) return tc_gemm_workspace_bytes(n, n, n, 6, true);
  return 0;
}

// FP64 / complex128 products on the INT8 tensor cores (Ozaki scheme): by
// default for products of at least kOzAutoMinDim in every dimension, where it
// measured faster than the FP64 tensor cores (2048^3: 405 against 551 us real,
// 1383 against 1856 us complex), with kOzAutoDigits digits (49 bits); a handle
// can turn it off or force it with a digit count (calamanSetDoubleEmulation).
inline constexpr int kOzAutoMinDim = 1536;
inline constexpr int kOzAutoDigits = 7;
inline constexpr int kOzForcedMinDim = 128;

template <typename T> inline int oz_digits_for(calamanHandle_t h, int n) {
  if (!std::is_same<T, double>::value && !std::is_same<T, double2>::value) return 0;
  const int d = h ? h->fp64_digits : -1;
  if (d == 0) return 0;
  const int digits = d < 0 ? kOzAutoDigits : d;
  const int min_dim = d < 0 ? kOzAutoMinDim : kOzForcedMinDim;
  if (n < min_dim || !oz_gemm_supported(n, elem<T>::complex, digits)) return 0;
  return digits;
}
template <typename T> inline int oz_min_dim_for(calamanHandle_t h) {
  return (h && h->fp64_digits > 0) ? kOzForcedMinDim : kOzAutoMinDim;
}
template <typename T> inline std::size_t oz_scratch_bytes(calamanHandle_t h, int n) {
  const int d = oz_digits_for<T>(h, n);
  return d ? oz_gemm_workspace_bytes(n, n, n, elem<T>::complex, d) : 0;
}

// The GEMM scratch a driver lends for one call: split-BF16 operand parts
// (FP32 tiers) and the emulated FP64 products' digit planes.
template <typename T>
inline GemmScratch lend_scratch(calamanHandle_t h, int n, void *tc, std::size_t tc_bytes, void *oz,
                         std::size_t oz_bytes) {
  GemmScratch gs;
  gs.ptr = tc;
  gs.bytes = tc_bytes;
  gs.terms = split_terms_of(h);
  gs.oz = oz;
  gs.oz_bytes = oz_bytes;
  gs.oz_digits = oz ? oz_digits_for<T>(h, n) : 0;
  gs.oz_min_dim = oz_min_dim_for<T>(h);
  return gs;
}

// The FP64 twin of a single-precision element type: the single tiers run
// their final squarings in FP64.
template <typename T> struct Wide { using type = T; };
template <> struct Wide<float> { using type = double; };
template <> struct Wide<float2> { using type = double2; };

struct PointerModeScope {  // save / force host / restore, src/expm/expm.cppm:107-115
  calamanHandle_t h;
  int saved;
  explicit PointerModeScope(calamanHandle_t handle) : h(handle), saved(CALAMAN_POINTER_MODE_HOST) {
    if (h) {
      saved = h->pointer_mode;
      h->pointer_mode = CALAMAN_POINTER_MODE_HOST;
    }
  }
  ~PointerModeScope() {
    if (h) h->pointer_mode = saved;
  }
};

}  // namespace clm
