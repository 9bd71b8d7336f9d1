// Construction of the device-resident tables of one modulus chain.
//
// Everything here is exact integer arithmetic on the host (unsigned __int128)
// followed by one upload; nothing runs per operation.  The NTT root choice
// follows the reference exactly (fhelium/engine/ntt/plans/twiddles.py:10-20:
// psi = the first c^((q-1)/2N), c = 2, 3, ..., whose N-th power is not 1),
// because NTT-domain residues are only comparable under the same psi.  The
// hybrid digit partition follows fhelium/engine/rns/decomposition.py:30-53
// (P-wide groups of scale primes, then the structural base prime alone;
// level l keeps the primes with id >= l).
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>

#include "fhb_context.h"

namespace fhb {

namespace {
thread_local std::string g_last_error;

using u128 = unsigned __int128;

uint64_t mulmod(uint64_t a, uint64_t b, uint64_t q) { return static_cast<uint64_t>((u128)a * b % q); }

uint64_t powmod(uint64_t b, uint64_t e, uint64_t q) {
  uint64_t r = 1 % q;
  b %= q;
  while (e) {
    if (e & 1) r = mulmod(r, b, q);
    b = mulmod(b, b, q);
    e >>= 1;
  }
  return r;
}

uint64_t invmod(uint64_t a, uint64_t q) { return powmod(a % q, q - 2, q); }  // q prime

uint64_t primitive_2nth_root(uint64_t q, uint64_t n) {
  const uint64_t e = (q - 1) / (2 * n);
  for (uint64_t c = 2; c < n; ++c) {
    const uint64_t r = powmod(c, e, q);
    if (powmod(r, n, q) != 1) return r;
  }
  return 0;
}

template <typename T>
T shoup_of(uint64_t w, uint64_t q) {
  if (sizeof(T) == 8) return static_cast<T>((((u128)w) << 64) / q);
  return static_cast<T>((((uint64_t)w) << 32) / q);
}

template <typename T>
TwPair<T> pair(uint64_t w, uint64_t q) {
  return TwPair<T>{static_cast<T>(w), shoup_of<T>(w, q)};
}

// -q^{-1} mod 2^bits by Newton iteration on odd q.
uint64_t neg_inv_pow2(uint64_t q, int bits) {
  uint64_t x = 1;
  for (int i = 0; i < 7; ++i) x *= 2 - q * x;
  const uint64_t mask = bits == 64 ? ~0ull : ((uint64_t{1} << bits) - 1);
  return (0 - x) & mask;
}

uint32_t bitrev(uint32_t v, int bits) {
  uint32_t r = 0;
  for (int i = 0; i < bits; ++i) {
    r = (r << 1) | (v & 1);
    v >>= 1;
  }
  return r;
}

template <typename T>
T* upload(Context& c, const std::vector<T>& host) {
  if (host.empty()) return nullptr;
  void* p = nullptr;
  if (cudaMalloc(&p, host.size() * sizeof(T)) != cudaSuccess) return nullptr;
  c.allocations.push_back(p);
  if (cudaMemcpy(p, host.data(), host.size() * sizeof(T), cudaMemcpyHostToDevice) != cudaSuccess)
    return nullptr;
  return static_cast<T*>(p);
}

// (prod of moduli[ids[0..k)]) mod m
uint64_t prefix_product_mod(const std::vector<uint64_t>& mods, int k, uint64_t m) {
  uint64_t r = 1 % m;
  for (int i = 0; i < k; ++i) r = mulmod(r, mods[i] % m, m);
  return r;
}

template <typename T>
bool build_tables(Context& c, ChainTables<T>& t, std::vector<LevelTables<T>>& levels, LevelTables<T>*& levels_dev) {
  const int qp = c.qp();
  const uint64_t n = c.n();
  const int radix_bits = sizeof(T) == 8 ? 62 : 30;
  const uint64_t R_mod = 0;  // placeholder to keep the intent explicit
  (void)R_mod;

  std::vector<PrimeInfo<T>> info(qp);
  std::vector<TwPair<T>> fwd(size_t(qp) * n), inv(size_t(qp) * n);
  c.roots.assign(qp, 0);
  for (int j = 0; j < qp; ++j) {
    const uint64_t q = c.moduli[j];
    const uint64_t r = powmod(2, radix_bits, q);  // R mod q
    const uint64_t rinv = invmod(r, q);
    const uint64_t ninv = invmod(n % q, q);
    PrimeInfo<T>& p = info[j];
    p.q = T(q);
    p.twice_q = T(2 * q);
    p.neg_inv = T(neg_inv_pow2(q, radix_bits));
    p.r2 = T(mulmod(r, r, q));
    p.rmod = T(r);
    p.rmod_s = shoup_of<T>(r, q);
    p.one_s = shoup_of<T>(1, q);
    p.ninv = T(ninv);
    p.ninv_s = shoup_of<T>(ninv, q);
    const uint64_t nr = mulmod(ninv, rinv, q);
    p.ninv_rinv = T(nr);
    p.ninv_rinv_s = shoup_of<T>(nr, q);
    p.rinv = T(rinv);
    p.rinv_s = shoup_of<T>(rinv, q);

    const uint64_t psi = primitive_2nth_root(q, n);
    if (psi == 0) return false;
    c.roots[j] = psi;
    const uint64_t psi_inv = invmod(psi, q);
    std::vector<uint64_t> pw(n), pwi(n);
    pw[0] = pwi[0] = 1;
    for (uint64_t i = 1; i < n; ++i) {
      pw[i] = mulmod(pw[i - 1], psi, q);
      pwi[i] = mulmod(pwi[i - 1], psi_inv, q);
    }
    for (uint64_t k = 0; k < n; ++k) {
      const uint32_t b = bitrev(uint32_t(k), c.log_n);
      fwd[size_t(j) * n + k] = pair<T>(pw[b], q);
      inv[size_t(j) * n + k] = pair<T>(pwi[b], q);
    }
  }
  t.prime = upload(c, info);
  t.tw_fwd = upload(c, fwd);
  t.tw_inv = upload(c, inv);
  // FP64 tables of the rows of primes below 2^42 (int64 chains whose leading
  // Q primes are that narrow; the rows of wider primes keep the integer
  // tables): the constants and the twiddles as (c, c / q) double pairs, and
  // the twiddles also as plain values (the standalone transforms' products
  // take the quotient from 1/q)
  bool f64 = false;
  if constexpr (sizeof(T) == 8) {
    c.f64_prime_end = 0;
    while (c.f64_prime_end < c.num_q && c.moduli[c.f64_prime_end] < (uint64_t{1} << 42)) ++c.f64_prime_end;
    f64 = c.f64_prime_end > 0;
    if (f64) {
      auto dpair = [](uint64_t w, uint64_t q) { return TwPair<double>{double(w), double(w) / double(q)}; };
      std::vector<PrimeInfo<double>> dinfo(qp);
      std::vector<TwPair<double>> dfwd(fwd.size(), TwPair<double>{0.0, 0.0}), dinv(inv.size(), TwPair<double>{0.0, 0.0});
      std::vector<double> vfwd(fwd.size(), 0.0), vinv(inv.size(), 0.0);
      for (int j = 0; j < qp; ++j) {
        const uint64_t q = c.moduli[j];
        const PrimeInfo<T>& p = info[j];
        PrimeInfo<double>& d = dinfo[j];
        d.q = double(q);
        d.twice_q = 2.0 * double(q);
        d.one_s = 1.0 / double(q);
        const TwPair<double> rm = dpair(uint64_t(p.rmod), q), ni = dpair(uint64_t(p.ninv), q),
                             nr = dpair(uint64_t(p.ninv_rinv), q), ri = dpair(uint64_t(p.rinv), q);
        d.rmod = rm.w, d.rmod_s = rm.wp, d.ninv = ni.w, d.ninv_s = ni.wp;
        d.ninv_rinv = nr.w, d.ninv_rinv_s = nr.wp, d.rinv = ri.w, d.rinv_s = ri.wp;
        if (j >= c.f64_prime_end) continue;
        for (uint64_t k = 0; k < n; ++k) {
          const size_t at = size_t(j) * n + k;
          dfwd[at] = dpair(uint64_t(fwd[at].w), q);
          dinv[at] = dpair(uint64_t(inv[at].w), q);
          vfwd[at] = dfwd[at].w;
          vinv[at] = dinv[at].w;
        }
      }
      c.t64f.prime = upload(c, dinfo);
      c.t64f.tw_fwd = upload(c, dfwd);
      c.t64f.tw_inv = upload(c, dinv);
      c.t64f.twv_fwd = upload(c, vfwd);
      c.t64f.twv_inv = upload(c, vinv);
    }
  }

  // ---- ModDown by P -------------------------------------------------------
  std::vector<uint64_t> pm(c.moduli.begin() + c.num_q, c.moduli.end());
  std::vector<TwPair<T>> pg(kMaxDigitWidth * kMaxDigitWidth, TwPair<T>{0, 0});
  for (int k = 0; k < c.num_p; ++k) {
    for (int i = 0; i < k; ++i) pg[k * kMaxDigitWidth + i] = pair<T>(prefix_product_mod(pm, i, pm[k]), pm[k]);
    pg[k * kMaxDigitWidth + k] = pair<T>(invmod(prefix_product_mod(pm, k, pm[k]), pm[k]), pm[k]);
  }
  std::vector<TwPair<T>> pmix(size_t(kMaxDigitWidth) * qp, TwPair<T>{0, 0}), pinv(qp, TwPair<T>{0, 0}),
      prinv(qp, TwPair<T>{0, 0});
  for (int pid = 0; pid < qp; ++pid) {
    const uint64_t m = c.moduli[pid];
    for (int k = 0; k < c.num_p; ++k) pmix[size_t(k) * qp + pid] = pair<T>(prefix_product_mod(pm, k, m), m);
    if (pid < c.num_q) {
      const uint64_t p_mod = prefix_product_mod(pm, c.num_p, m);
      pinv[pid] = pair<T>(invmod(p_mod, m), m);
      prinv[pid] = pair<T>(mulmod(p_mod, invmod(powmod(2, radix_bits, m), m), m), m);
    }
  }
  t.p_garner = upload(c, pg);
  t.p_mix = upload(c, pmix);
  t.p_inv = upload(c, pinv);
  t.p_rinv = upload(c, prinv);
  if (f64) {
    // the FP64 core's relinearisation addend P c R: P mod q (not P R^{-1})
    std::vector<TwPair<double>> dp(qp, TwPair<double>{0.0, 0.0});
    for (int pid = 0; pid < c.f64_prime_end; ++pid) {
      const uint64_t m = c.moduli[pid], p_mod = prefix_product_mod(pm, c.num_p, m);
      dp[pid] = TwPair<double>{double(p_mod), double(p_mod) / double(m)};
    }
    c.t64f.p_rinv = upload(c, dp);
    c.f64_tables_ok = c.t64f.prime && c.t64f.tw_fwd && c.t64f.tw_inv && c.t64f.twv_fwd && c.t64f.twv_inv &&
                      c.t64f.p_rinv;
  }

  // ---- per level: hybrid digits, Garner and extension constants, rescale --
  std::vector<std::vector<int>> level0;
  for (int s = 0; s < c.num_q - 1; s += c.num_p) {
    std::vector<int> d;
    for (int i = s; i < std::min(s + c.num_p, c.num_q - 1); ++i) d.push_back(i);
    level0.push_back(d);
  }
  level0.push_back({c.num_q - 1});
  levels.assign(c.num_q, LevelTables<T>{});
  c.level_digits.assign(c.num_q, {});
  const int d0 = int(level0.size());
  std::vector<TwPair<double>> ext64f;
  if (f64) ext64f.assign(size_t(c.num_q) * d0 * kMaxDigitWidth * 2 * qp, TwPair<double>{0.0, 0.0});
  for (int level = 0; level < c.num_q; ++level) {
    LevelTables<T>& lt = levels[level];
    std::vector<DigitDesc> dd;
    std::vector<TwPair<T>> gar, ext;
    for (int kd = 0; kd < int(level0.size()); ++kd) {
      std::vector<uint64_t> b;
      int first = -1;
      for (int pid : level0[kd])
        if (pid >= level) {
          if (first < 0) first = pid;
          b.push_back(c.moduli[pid]);
        }
      if (b.empty()) continue;
      const int alpha = int(b.size());
      dd.push_back(DigitDesc{first, alpha, kd, 0});
      std::vector<TwPair<T>> g(kMaxDigitWidth * kMaxDigitWidth, TwPair<T>{0, 0});
      for (int k = 0; k < alpha; ++k) {
        for (int i = 0; i < k; ++i) g[k * kMaxDigitWidth + i] = pair<T>(prefix_product_mod(b, i, b[k]), b[k]);
        g[k * kMaxDigitWidth + k] = pair<T>(invmod(prefix_product_mod(b, k, b[k]), b[k]), b[k]);
      }
      gar.insert(gar.end(), g.begin(), g.end());
      std::vector<TwPair<T>> e(size_t(kMaxDigitWidth) * qp, TwPair<T>{0, 0});
      for (int r = 0; r < alpha; ++r)
        for (int pid = 0; pid < qp; ++pid) e[size_t(r) * qp + pid] = pair<T>(prefix_product_mod(b, r, c.moduli[pid]), c.moduli[pid]);
      ext.insert(ext.end(), e.begin(), e.end());
      if (f64) {
        const int a = int(dd.size()) - 1;
        for (int r = 0; r < alpha; ++r)
          for (int pid = 0; pid < c.f64_prime_end; ++pid) {
            const uint64_t m = c.moduli[pid], cr = prefix_product_mod(b, r, m);
            const size_t at = ((((size_t(level) * d0 + a) * kMaxDigitWidth + r) * 2) * qp) + pid;
            const uint64_t hi = mulmod(cr, (uint64_t{1} << 30) % m, m);
            ext64f[at] = TwPair<double>{double(hi), double(hi) / double(m)};
            ext64f[at + qp] = TwPair<double>{double(cr), double(cr) / double(m)};
          }
      }
    }
    lt.num_digits = int(dd.size());
    c.level_digits[level] = dd;
    lt.digits = upload(c, dd);
    lt.garner = upload(c, gar);
    lt.ext = upload(c, ext);
    std::vector<TwPair<T>> rs(qp, TwPair<T>{0, 0});
    const uint64_t qd = c.moduli[level];
    for (int pid = 0; pid < qp; ++pid)
      if (pid != level) rs[pid] = pair<T>(invmod(qd % c.moduli[pid], c.moduli[pid]), c.moduli[pid]);
    lt.rescale_inv = upload(c, rs);
    if (!lt.digits || !lt.garner || !lt.ext || !lt.rescale_inv) return false;
  }
  levels_dev = upload(c, levels);
  if (!levels_dev) return false;
  if (f64) {
    c.ext64f = upload(c, ext64f);
    c.ext64f_digits = d0;
    c.f64_tables_ok = c.f64_tables_ok && c.ext64f;
  }
  return t.prime && t.tw_fwd && t.tw_inv && t.p_garner && t.p_mix && t.p_inv && t.p_rinv;
}

}  // namespace

void set_error(const std::string& msg) { g_last_error = msg; }
const char* last_error() { return g_last_error.c_str(); }

int fail(int code, const std::string& msg) {
  set_error(msg);
  return code;
}

int ensure_dynamic_smem(const void* kernel, int bytes) {
  static std::mutex mu;
  static std::vector<std::pair<std::pair<int, const void*>, int>> done;
  int device = 0;
  cudaGetDevice(&device);
  std::lock_guard<std::mutex> lock(mu);
  for (const auto& e : done)
    if (e.first.first == device && e.first.second == kernel && e.second >= bytes) return 0;
  cudaError_t e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
  if (e != cudaSuccess) return cuda_status(e, "cudaFuncSetAttribute");
  done.push_back({{device, kernel}, bytes});
  return 0;
}

int cuda_status(cudaError_t e, const char* where) {
  if (e == cudaSuccess) return 0;
  set_error(std::string(where) + ": " + cudaGetErrorString(e));
  return 1000 + int(e);
}

Context* build_context(int bits, int log_n, const uint64_t* moduli, int num_q, int num_p, int device,
                       int* status) {
  Context* c = new Context();
  c->bits = bits;
  c->log_n = log_n;
  c->num_q = num_q;
  c->num_p = num_p;
  c->device = device;
  c->moduli.assign(moduli, moduli + num_q + num_p);
  bool ok = bits == 64 ? build_tables<uint64_t>(*c, c->t64, c->lv64, c->lv64_dev)
                       : build_tables<uint32_t>(*c, c->t32, c->lv32, c->lv32_dev);
  if (!ok) {
    cudaError_t e = cudaGetLastError();
    *status = e != cudaSuccess ? cuda_status(e, "context tables") : fail(-3, "no primitive 2N-th root for a modulus");
    for (void* p : c->allocations) cudaFree(p);
    delete c;
    return nullptr;
  }
  *status = 0;
  return c;
}

void destroy_context(Context* c) {
  if (!c) return;
  int prev = 0;
  cudaGetDevice(&prev);
  cudaSetDevice(c->device);
  for (void* p : c->allocations) cudaFree(p);
  for (cudaStream_t s : c->ov_streams)
    if (s) cudaStreamDestroy(s);
  for (cudaEvent_t e : c->ov_events) cudaEventDestroy(e);
  cudaSetDevice(prev);
  delete c->tc;
  delete c->tcb;
  delete c;
}

}  // namespace fhb
