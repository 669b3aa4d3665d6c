// Compiles a reference-style call site against include/calaman_b200.hpp and
// runs the host-only contracts (no device work): the plan ladder, the
// Paterson-Stockmeyer cost table, buffer sizes and argument rejection
// (test/expm/expm_tests.cpp:389-465, test/paterson_stockmeyer/paterson_stockmeyer_tests.cpp:235-383).
#include <cstdio>
#include <string>
#include <vector>

#include "calaman_b200.hpp"

#define CHECK(c)                                              \
  do {                                                        \
    if (!(c)) {                                               \
      std::printf("FAILED %s:%d %s\n", __FILE__, __LINE__, #c); \
      return 1;                                               \
    }                                                         \
  } while (0)

int main() {
  // plan ladder
  const int want[5] = {2, 3, 4, 5, 6};
  const int deg[5] = {3, 5, 7, 9, 13};
  for (int i = 0; i < 5; ++i) {
    const calaman::ExpmPlan p = calaman::expm_plan<double>(calaman::pade_theta<double>(deg[i]) * 0.99);
    CHECK(p.s == 0 && p.m <= deg[i]);
    CHECK(p.num_gemms == want[p.m == 3 ? 0 : p.m == 5 ? 1 : p.m == 7 ? 2 : p.m == 9 ? 3 : 4]);
  }
  const calaman::ExpmPlan big = calaman::expm_plan<float>(calaman::pade_theta<float>(13) * 40.f);
  CHECK(big.m == 13 && big.s > 0 && big.num_gemms == 6 + big.s);
  CHECK(calaman::pade_theta<double>(4) == 0.0);

  // PS cost table
  CHECK(calaman::paterson_stockmeyer_plan(4).num_gemms == 3);
  CHECK(calaman::paterson_stockmeyer_plan(30).num_gemms == 10);
  const auto p12 = calaman::paterson_stockmeyer_plan(12);
  CHECK(p12.s == 3 && p12.num_gemms == 6 && p12.num_blocks == 3);
  CHECK(calaman::paterson_stockmeyer_bufferSize<double>(10, 1) == 0);

  // argument rejection before any device work (null handles, host pointers)
  const int n = 4;
  std::vector<double> a(n * n, 1.0), e(n * n, 0.0), work(64, 0.0);
  int info[2] = {0, 0};
  auto call = [&](int nn, int lda, int lde, void *w) {
    return calaman::expm<double>(nullptr, nullptr, nullptr, nn, a.data(), lda, e.data(), lde, w,
                                 work.size() * sizeof(double), info);
  };
  const calaman::Status invalid{calamanStatus_t{CALAMAN_DOMAIN_BLAS, CALAMAN_STATUS_INVALID_VALUE}};
  CHECK(call(0, n, n, work.data()) == invalid);
  CHECK(call(n, n - 1, n, work.data()) == invalid);
  CHECK(call(n, n, n - 1, work.data()) == invalid);
  CHECK(call(n, n, n, nullptr) == invalid);
  CHECK(!call(n, n, n, work.data()).ok());  // undersized workspace
  std::size_t bytes = 0;
  CHECK(calaman::expm_bufferSize<std::complex<double>>(nullptr, 8, &bytes).ok() && bytes > 0);
  CHECK(!calaman::pade_bufferSize<float>(nullptr, 6, 4, &bytes).ok());

  std::vector<double> c(5, 1.0), p(n * n, 0.0);
  const calaman::Status st = calaman::horner<double>(nullptr, 0, c.data(), 4, a.data(), n, p.data(), n,
                                                     work.data(), 4096);
  CHECK(st.code == CALAMAN_STATUS_NOT_INITIALIZED && std::string(st.name()) == "NOT_INITIALIZED");
  // the new entries: size queries and argument rejection
  CHECK(calaman::expm_vjp_bufferSize<double>(nullptr, 8, &bytes).ok() && bytes > 0);
  std::vector<double> g(n * n, 0.5), d(n * n, 0.0);
  CHECK(calaman::expm_vjp<double>(nullptr, nullptr, nullptr, 0, a.data(), n, g.data(), n, d.data(), n, nullptr,
                                  n, work.data(), 4096, info) == invalid);
  const int ns[3] = {4, 16, 300};
  CHECK(calaman::expm_batched_bufferSize<float>(nullptr, 2, ns, &bytes).ok() && bytes > 0);
  CHECK(calaman::expm_batched_bufferSize<float>(nullptr, 3, ns, &bytes).code == CALAMAN_STATUS_NOT_SUPPORTED);
  CHECK(calaman::expm_vjp_batched_bufferSize<double>(nullptr, 2, ns, &bytes).ok() && bytes > 0);
  CHECK(calaman::expm_batched<double>(nullptr, nullptr, nullptr, 0, ns, nullptr, nullptr, nullptr, nullptr,
                                      nullptr, 0, nullptr).ok());  // an empty batch is a no-op
  int lw = 0, ilo = 0, ihi = 0;
  CHECK(calaman::gebal_bufferSize<double>(8, &lw).ok() && lw >= 1);
  CHECK(calaman::gebal<double>(nullptr, calaman::GebalJob::Permute, 4, a.data(), 4, &ilo, &ihi, work.data(),
                               &lw).code == CALAMAN_STATUS_NOT_SUPPORTED);
  CHECK(calaman::expm_balanced_bufferSize<std::complex<float>>(nullptr, 16, &bytes).ok() && bytes > 0);
  // expm_herm / heevd: size queries and host-side rejection
  CHECK(calaman::expm_herm_bufferSize<std::complex<double>>(nullptr, calaman::FillMode::Upper, 16, &bytes).ok() &&
        bytes > 0);
  CHECK(calaman::heevd_bufferSize<float>(calaman::FillMode::Lower, 16, &bytes).ok() && bytes > 0);
  CHECK(calaman::expm_herm<double>(nullptr, nullptr, nullptr, calaman::FillMode::Lower, 0, a.data(), n, d.data(), n,
                                   work.data(), 4096, info) == invalid);
  // geodesic trial points: size query and rejection
  CHECK(calaman::geodesic_points_bufferSize<std::complex<double>>(nullptr, 32, 6, &bytes).ok() && bytes > 0);
  CHECK(calaman::geodesic_points_bufferSize<double>(nullptr, 32, 65, &bytes) == invalid);
  // lacn2: size query and host-side rejection (no device work)
  CHECK(calaman::lacn2_bufferSize<double>(100) >= 100 * sizeof(int));
  double est = 0;
  int kase = 1;
  std::array<int, 3> isave{9, 0, 0};
  CHECK(calaman::lacn2<double>(nullptr, 4, d.data(), g.data(), work.data(), 1 << 20, est, kase, isave) == invalid);
  std::printf("header_check ok\n");
  return 0;
}
