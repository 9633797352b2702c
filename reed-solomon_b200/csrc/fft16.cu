// Host side of the ReedSolomon16 FFT route: program construction (fft16.hpp) and the
// launch sequence of one run.
#include "fft16.hpp"

#include <algorithm>

#include "gf_host.hpp"
#include "kernels_fft16.cuh"
#include "runtime.hpp"

namespace rsb {

namespace {

// WHAT[l][x] of the tower field: W_0(x) = x, W_{j+1}(x) = W_j(x) (W_j(x) + W_j(2^j)),
// each level scaled so that W_l(2^l) = 1 (src/fft16.rs:42-70). Evaluated per point by
// running the recurrence, which needs the unscaled pivots W_j(2^j).
struct What16 {
  uint16_t pivot[16], pivot_inv[16];
  What16() {
    for (int l = 0; l < 16; l++) {
      pivot[l] = raw(l, (uint16_t)(1u << l));
      pivot_inv[l] = gf16_inv(pivot[l]);
    }
  }
  uint16_t raw(int l, uint16_t x) const {
    uint16_t w = x;
    for (int j = 0; j < l; j++) w = gf16_mul(w, (uint16_t)(w ^ pivot[j]));
    return w;
  }
  uint16_t operator()(int l, uint16_t x) const { return gf16_mul(raw(l, x), pivot_inv[l]); }
};

const What16 &what16() {
  static const What16 w;
  return w;
}

int log2_exact(uint64_t x) {
  int l = 0;
  while ((1ull << l) < x) l++;
  return l;
}

// Table entry of a tower constant c (16 u16): the column bytes k_t * 2^p (p = 0..7) of
// its Karatsuba factors k0 = c_lo, k1 = c_hi + c_lo, k2 = 32 c_hi, then 8 zero bytes.
// Column words of GF(2^8) constants: for each a, the u16 pairs (a * 2^(2w)) |
// (a * 2^(2w+1)) << 8 for w = 0..3, by repeated doubling modulo x^8+x^4+x^3+x^2+1.
struct ColumnWords {
  uint16_t w[256][4];
  ColumnWords() {
    for (int a = 0; a < 256; a++) {
      uint8_t v = (uint8_t)a, b[8];
      for (int q = 0; q < 8; q++) {
        b[q] = v;
        v = (uint8_t)((v << 1) ^ ((v & 0x80) ? 0x1d : 0));
      }
      for (int i = 0; i < 4; i++) w[a][i] = (uint16_t)(b[2 * i] | (b[2 * i + 1] << 8));
    }
  }
};

void push_const16(std::vector<uint16_t> &cols, uint16_t c) {
  static const ColumnWords cw;
  const uint8_t hi = (uint8_t)(c >> 8), lo = (uint8_t)c;
  const uint8_t k[3] = {lo, (uint8_t)(hi ^ lo), gf8_mul(hi, 32)};
  const size_t at = cols.size();
  cols.resize(at + 16);  // three factors' 4 words each, then the factors, then zeros
  uint16_t *o = cols.data() + at;
  for (int t = 0; t < 3; t++)
    for (int i = 0; i < 4; i++) o[t * 4 + i] = cw.w[k[t]][i];
  o[12] = (uint16_t)(k[0] | (k[1] << 8));  // bytes 24..26: k0, k1, k2
  o[13] = k[2];
}

uint64_t push_const(Fft16Program &p, uint16_t c) {
  uint64_t at = p.cols.size() / 16;
  push_const16(p.cols, c);
  return at;
}

// f(WHAT_l(beta ^ (j << (l + 1)))) for j = 0 .. count-1. WHAT_l is a normalised
// subspace polynomial, which is GF(2)-linear, so consecutive values differ by the XOR of
// its values on the low bits that flip from j-1 to j: one multiply chain per basis bit
// instead of l multiplies per constant.
template <class F>
void for_level_consts(int l, uint32_t beta, uint32_t count, F &&f) {
  const What16 &w = what16();
  uint16_t flip[16];  // flip[t] = XOR of WHAT_l(2^(i + l + 1)) for i <= t
  uint16_t acc = 0;
  for (int i = 0; i < 16 && (1u << i) < count; i++) flip[i] = acc ^= w(l, (uint16_t)(1u << (i + l + 1)));
  uint16_t v = w(l, (uint16_t)beta);
  f(v);
  for (uint32_t j = 1; j < count; j++) {
    v ^= flip[__builtin_ctz(j)];
    f(v);
  }
}

// Constants of a transform of `size` registers at `beta`: (l, j) at size - (size >> l) + j.
uint64_t push_transform(Fft16Program &p, uint32_t size, uint32_t beta) {
  uint64_t at = p.cols.size() / 16;
  const int lg = log2_exact(size);
  for (int l = 0; l < lg; l++) for_level_consts(l, beta, size >> (l + 1), [&](uint16_t c) { push_const(p, c); });
  p.butterflies += (uint64_t)(size / 2) * lg;
  return at;
}

void transform(Fft16Program &p, uint8_t src_buf, uint32_t src_start, uint8_t dst_buf, uint32_t dst_start,
               uint32_t size, uint32_t beta, bool inverse) {
  Fft16Step s{};
  s.kind = Fft16Step::kTransform;
  s.src_buf = src_buf;
  s.dst_buf = dst_buf;
  s.src_start = src_start;
  s.dst_start = dst_start;
  s.size = size;
  s.inverse = inverse;
  s.cols = push_transform(p, size, beta);
  p.interp.push_back(s);
}

void mulxor(Fft16Program &p, uint8_t src_buf, uint32_t src_start, uint32_t dst_start, uint32_t count, uint16_t c) {
  if (c == 0 || count == 0) return;
  Fft16Step s{};
  s.kind = Fft16Step::kMulXor;
  s.src_buf = src_buf;
  s.dst_buf = 0;
  s.src_start = src_start;
  s.dst_start = dst_start;
  s.size = count;
  s.cols = c == 1 ? Fft16Program::kNoConst : push_const(p, c);
  p.butterflies += count;
  p.interp.push_back(s);
}

// Builder::interpolate (src/fft.rs:198-239) on C registers [start, start+n): the first k
// hold values at beta + 0 .. beta + k-1; afterwards they hold the novel-basis
// coefficients (the rest stay zero).
void interpolate(Fft16Program &p, uint32_t start, uint32_t n, uint32_t beta, uint32_t k) {
  if (k == n) {
    if (n > 1) transform(p, 0, start, 0, start, n, beta, true);
    return;
  }
  const uint32_t half = n / 2;
  if (k <= half) {
    interpolate(p, start, half, beta, k);
    return;
  }
  if (half > 1) transform(p, 0, start, 0, start, half, beta, true);
  const uint16_t c = what16()(log2_exact(n) - 1, (uint16_t)beta);
  // Evaluate the first half's polynomial on the second half's points (in S), subtract.
  if (half > 1) {
    transform(p, 0, start, 1, 0, half, beta ^ half, false);
    mulxor(p, 1, 0, start + half, k - half, 1);
    p.uses_s = true;
  } else {
    mulxor(p, 0, start, start + half, k - half, 1);
  }
  interpolate(p, start + half, half, beta ^ half, k - half);
  mulxor(p, 0, start + half, start, k - half, c);
}

}  // namespace

bool fft16_build(size_t k, size_t m, Fft16Program &p) {
  if (k < 2 || m == 0 || k + m > 65536) return false;
  p = Fft16Program{};
  p.k = (uint32_t)k;
  p.m = (uint32_t)m;
  uint32_t t = 1;
  while (t < k) t <<= 1;
  p.t = t;
  // Constants: interpolation transforms of t, t/2, ... registers (fewer than 2t), one
  // per mulxor (at most log t) and t per evaluation coset (at most (k+m)/t + 1).
  p.cols.reserve((size_t)16 * ((size_t)t * (3 + (k + m) / t) + 32));
  interpolate(p, 0, t, 0, (uint32_t)k);
  const uint64_t n = k + m;
  for (uint64_t beta = 0; beta < n; beta += t) {
    const uint64_t lo = std::max<uint64_t>(k, beta), hi = std::min<uint64_t>(n, beta + t);
    if (lo >= hi) continue;
    Fft16Eval e{};
    e.beta = (uint32_t)beta;
    e.cols = push_transform(p, t, (uint32_t)beta);
    e.r_lo = (uint32_t)(lo - beta);
    e.r_hi = (uint32_t)(hi - beta);
    e.parity_row = lo - k;
    p.evals.push_back(e);
  }
  p.eval_in_place = p.evals.size() == 1;
  if (p.cols.capacity() > p.cols.size() + p.cols.size() / 2) p.cols.shrink_to_fit();
  return true;
}

bool fft16_decode_build(size_t k, size_t m, const std::vector<uint32_t> &survivors,
                        const std::vector<uint32_t> &targets, Fft16Decode &d) {
  const size_t n = k + m;
  if (k < 1 || n > 65536 || survivors.size() != k || targets.empty()) return false;
  d = Fft16Decode{};
  d.n = (uint32_t)n;
  uint32_t N = 2;
  while (N < n) N <<= 1;
  d.N = N;
  d.lg = (uint32_t)log2_exact(N);
  d.targets = targets;
  // Log-domain XOR-convolution conv[x] = sum_{e in E} log(x ^ e) (log 0 taken as 0),
  // by Walsh-Hadamard transforms in wrapping 64-bit arithmetic: the true sums are
  // below 2^32 and N <= 2^16, so N * conv is exact modulo 2^64.
  const Gf16Tables &T = gf16();
  std::vector<uint64_t> a(N, 1), b(N, 0);
  for (uint32_t s : survivors) a[s] = 0;
  for (uint32_t x = 1; x < N; x++) b[x] = T.log[x];
  auto fwht = [N](std::vector<uint64_t> &v) {
    for (uint32_t h = 1; h < N; h <<= 1)
      for (uint32_t i = 0; i < N; i += 2 * h)
        for (uint32_t j = i; j < i + h; j++) {
          const uint64_t x = v[j], y = v[j + h];
          v[j] = x + y;
          v[j + h] = x - y;
        }
  };
  fwht(a);
  fwht(b);
  for (uint32_t x = 0; x < N; x++) a[x] *= b[x];
  fwht(a);
  auto locator = [&](uint32_t x) { return T.exp[(a[x] / N) % 65535]; };
  auto push16 = [&](uint16_t c) { push_const16(d.cols, c); };
  d.cols.reserve((size_t)16 * (2 * N + d.lg + targets.size()));
  // Transform constants (beta 0, both directions): (l, j) at N - (N >> l) + j.
  for (uint32_t l = 0; l < d.lg; l++) for_level_consts((int)l, 0, N >> (l + 1), push16);
  // Row scales: L at the survivors, 0 elsewhere.
  d.row_off = d.cols.size() / 16;
  std::vector<uint16_t> scale(N, 0);
  for (uint32_t s : survivors) scale[s] = locator(s);
  for (uint32_t x = 0; x < N; x++) push16(scale[x]);
  // kappa_t = (product of the nonzero points of V_t) / W_t(2^t), since
  // W_t(x) = x * prod_{a in V_t, a != 0} (x - a).
  d.kappa_off = d.cols.size() / 16;
  uint64_t log_prod = 0;  // in the log domain: prod = exp(log_prod)
  for (uint32_t t = 0; t < d.lg; t++) {
    push16(gf16_mul(T.exp[log_prod % 65535], what16().pivot_inv[t]));
    for (uint32_t x = (1u << t); x < (2u << t); x++) log_prod += T.log[x];
  }
  // Target scales: 1 / L'(e) = exp(-log L'(e)).
  d.target_off = d.cols.size() / 16;
  for (uint32_t e : targets) push16(T.exp[(65535 - (a[e] / N) % 65535) % 65535]);
  d.butterflies = (uint64_t)3 * (N / 2) * d.lg + N + targets.size();
  return true;
}

bool fft16_decode_preferred(const Fft16Decode &d, size_t k) {
  // LOP3 per 32-symbol group: a butterfly or scaled row about 290, counted twice for
  // the passes' L2 traffic; the matrix route 208 per coefficient plus about as much
  // again to build its rows.
  const double fft = 2.0 * 290.0 * (double)d.butterflies;
  const double matrix = 2.0 * 208.0 * (double)d.targets.size() * k;
  return fft < matrix;
}

size_t fft16_decode_scratch_bytes(const Fft16Decode &d, size_t len, size_t budget) {
  const uint64_t G = (len / 2 + 31) / 32, per_group = (uint64_t)d.regs() * 64;
  return (size_t)std::max<uint64_t>(per_group, std::min<uint64_t>(G * per_group, budget / per_group * per_group));
}

int fft16_decode_run(const Fft16Decode &d, const uint16_t *d_cols, uint8_t *scratch, size_t scratch_bytes,
                     uint8_t *const *d_ptrs, const uint32_t *d_targets, size_t n_targets, size_t len,
                     cudaStream_t st) {
  if (n_targets == 0) return RS_OK;
  const uint32_t N = d.N;
  const uint64_t Nsym = len / 2, G = (Nsym + 31) / 32, per_group = (uint64_t)d.regs() * 64;
  if (scratch_bytes < per_group) return RS_ERR_TOO_LARGE;
  const uint64_t gc = std::min<uint64_t>(G, scratch_bytes / per_group);
  for (uint64_t g0 = 0; g0 < G; g0 += gc) {
    const uint64_t gn = std::min<uint64_t>(gc, G - g0);
    uint32_t *C = reinterpret_cast<uint32_t *>(scratch), *W = C + (uint64_t)N * gn * 16;
    const unsigned rthreads = (unsigned)std::min<uint64_t>(kFft16Threads, (gn + 31) / 32 * 32);
    const bool rt = fft16_rt();
    if (rt)
      fft16_scale_load_kernel<true><<<N, rthreads, 0, st>>>(d_ptrs, d_cols + d.row_off * 16, d.n, Nsym, g0, gn, C);
    else
      fft16_scale_load_kernel<false><<<N, rthreads, 0, st>>>(d_ptrs, d_cols + d.row_off * 16, d.n, Nsym, g0, gn, C);
    g_launches++;
    RSB_CU(cudaGetLastError());
    // Transforms of N registers at beta 0: inverse on C (levels 0, 1 | 2, 3 | ..., an
    // odd top level alone); the forward one on W mirrors it.
    auto pass = [&](uint32_t *buf, int level, int lv, bool inverse) -> int {
      Fft16PassArgs a{};
      a.src = buf;
      a.dst = buf;
      a.cols = d_cols;
      a.R = N;
      a.level = (uint32_t)level;
      a.src_regs = a.dst_regs = N;
      a.G = gn;
      a.n_stripes = 1;
      a.inverse = inverse;
      g_launches++;
      RSB_CU(launch_fft16_pass(a, lv, st));
      return RS_OK;
    };
    const int lg = (int)d.lg;
    int plan[40][2];
    const int np_inv = fft16_passes(lg, true, plan);
    for (int i = 0; i < np_inv; i++) RSB_TRY(pass(C, plan[i][0], plan[i][1], true));
    if (rt)
      fft16_derivative_kernel<true><<<N, rthreads, 0, st>>>(C, W, d_cols + d.kappa_off * 16, d.lg, gn);
    else
      fft16_derivative_kernel<false><<<N, rthreads, 0, st>>>(C, W, d_cols + d.kappa_off * 16, d.lg, gn);
    g_launches++;
    RSB_CU(cudaGetLastError());
    const int np_fwd = fft16_passes(lg, false, plan);
    for (int i = 0; i < np_fwd; i++) RSB_TRY(pass(W, plan[i][0], plan[i][1], false));
    const unsigned nt = (unsigned)std::min(n_targets, d.targets.size());
    if (rt)
      fft16_scale_store_kernel<true><<<nt, rthreads, 0, st>>>(W, d_targets, d_cols + d.target_off * 16, d_ptrs, Nsym,
                                                            g0, gn);
    else
      fft16_scale_store_kernel<false><<<nt, rthreads, 0, st>>>(W, d_targets, d_cols + d.target_off * 16, d_ptrs, Nsym,
                                                             g0, gn);
    g_launches++;
    RSB_CU(cudaGetLastError());
  }
  return RS_OK;
}

bool fft16_preferred(const Fft16Program &p) {
  // LOP3 per 32-symbol group: the matrix kernel about 208 per coefficient, a butterfly
  // about 290; the FFT's passes also move scratch through L2 (counted as 2x).
  const double fft = 2.0 * 290.0 * (double)p.butterflies + 64.0 * p.regs();
  const double matrix = 208.0 * (double)p.k * p.m;
  return fft < matrix;
}

static double fft16_time_us(const Fft16Program &p, size_t len, size_t n_stripes) {
  auto passes = [](uint64_t size) {
    int lg = 0, plan[40][2];
    while ((1ull << lg) < size) lg++;
    return (uint64_t)fft16_passes(lg, true, plan);
  };
  uint64_t launches = 1 + (p.k < p.t ? 1 : 0);  // load (+ zeroing)
  for (const Fft16Step &s : p.interp) launches += s.kind == Fft16Step::kTransform ? passes(s.size) : 1;
  launches += p.evals.size() * (passes(p.t) + 1);  // transform + store per coset
  const double groups = (double)n_stripes * (double)((len / 2 + 31) / 32);
  return 5.2 * (double)launches + 6.5e-5 * (double)p.butterflies * groups;
}

bool fft16_faster(const Fft16Program &p, size_t len, size_t n_stripes) {
  const double work = (double)p.k * (double)p.m * (double)len * (double)n_stripes;
  const double t_matrix = 2.0 + std::max(1.07 * (double)p.k, 4.6e-7 * work);
  return fft16_time_us(p, len, n_stripes) < t_matrix;
}

bool fft16_faster_than_gf8_matrix(const Fft16Program &p, size_t len, size_t n_stripes) {
  const double work = (double)p.k * (double)p.m * (double)len * (double)n_stripes;
  const double t_matrix = 2.0 + std::max(0.61 * (double)p.k, 2.0e-7 * work);
  return fft16_time_us(p, len, n_stripes) < t_matrix;
}

size_t fft16_scratch_bytes(const Fft16Program &p, size_t n_stripes, size_t len, size_t budget) {
  const uint64_t G = (len / 2 + 31) / 32, per_group = (uint64_t)p.regs() * 64;
  const uint64_t all = (uint64_t)n_stripes * G * per_group;
  return (size_t)std::max<uint64_t>(per_group, std::min<uint64_t>(all, budget / per_group * per_group));
}

int fft16_run(const Fft16Program &p, const uint16_t *d_cols, uint8_t *scratch, size_t scratch_bytes,
              const uint8_t *in_base, uint64_t in_row, uint64_t in_stripe, uint8_t *out_base, uint64_t out_row,
              uint64_t out_stripe, uint8_t *const *d_ptrs, size_t n_stripes, size_t len, cudaStream_t st) {
  const uint32_t t = p.t, k = p.k;
  const uint64_t N = len / 2, G = (N + 31) / 32, per_group = (uint64_t)p.regs() * 64;
  if (scratch_bytes < per_group) return RS_ERR_TOO_LARGE;
  // A unit of work: `wave` stripes x `gc` groups.
  uint64_t wave, gc;
  if (G * per_group <= scratch_bytes) {
    gc = G;
    wave = std::max<uint64_t>(1, std::min<uint64_t>(n_stripes, scratch_bytes / (G * per_group)));
  } else {
    wave = 1;
    gc = scratch_bytes / per_group;
  }
  const uint32_t regs_of[3] = {t, p.regs_s(), p.eval_in_place ? t : p.regs_w()};
  auto grid_for = [](uint64_t items) {
    return (unsigned)std::max<uint64_t>(1, std::min<uint64_t>((items + kFft16Threads - 1) / kFft16Threads, 148 * 16));
  };
  for (uint64_t s0 = 0; s0 < n_stripes; s0 += wave) {
    const uint32_t ns = (uint32_t)std::min<uint64_t>(wave, n_stripes - s0);
    for (uint64_t g0 = 0; g0 < G; g0 += gc) {
      const uint64_t gn = std::min<uint64_t>(gc, G - g0);
      uint32_t *buf[3];
      buf[0] = reinterpret_cast<uint32_t *>(scratch);
      buf[1] = buf[0] + (uint64_t)ns * regs_of[0] * gn * 16;
      buf[2] = p.eval_in_place ? buf[0] : buf[1] + (uint64_t)ns * regs_of[1] * gn * 16;
      auto pass = [&](const Fft16Step &s, const uint32_t *src, uint32_t src_regs, uint32_t src_start, int level,
                      int lv) -> int {
        Fft16PassArgs a{};
        a.src = src;
        a.dst = buf[s.dst_buf];
        a.cols = d_cols + s.cols * 16;
        a.R = s.size;
        a.level = (uint32_t)level;
        a.src_regs = src_regs;
        a.src_start = src_start;
        a.dst_regs = regs_of[s.dst_buf];
        a.dst_start = s.dst_start;
        a.G = gn;
        a.n_stripes = ns;
        a.inverse = s.inverse;
        g_launches++;
        RSB_CU(launch_fft16_pass(a, lv, st));
        return RS_OK;
      };
      // Levels of a transform: inverse 0, 1 | 2, 3 | ... (an odd top level alone, last);
      // forward the mirror image. The first pass reads the source window.
      auto run_transform = [&](const Fft16Step &s) -> int {
        const int lg = log2_exact(s.size);
        const uint32_t *src = buf[s.src_buf];
        uint32_t src_regs = regs_of[s.src_buf], src_start = s.src_start;
        auto advance = [&]() {
          src = buf[s.dst_buf];
          src_regs = regs_of[s.dst_buf];
          src_start = s.dst_start;
        };
        int plan[40][2];
        const int np = fft16_passes(lg, s.inverse != 0, plan);
        for (int i = 0; i < np; i++) {
          RSB_TRY(pass(s, src, src_regs, src_start, plan[i][0], plan[i][1]));
          advance();
        }
        return RS_OK;
      };
      // Data into C[0, k); C[k, t) zero.
      fft16_load_kernel<<<grid_for((uint64_t)ns * k * gn), kFft16Threads, 0, st>>>(
          in_base + s0 * in_stripe, in_row, in_stripe, reinterpret_cast<const uint8_t *const *>(d_ptrs), k, N, g0,
          gn, ns, t, buf[0]);
      g_launches++;
      RSB_CU(cudaGetLastError());
      if (k < t)
        RSB_CU(cudaMemset2DAsync(buf[0] + (uint64_t)k * gn * 16, (size_t)t * gn * 64, 0, (size_t)(t - k) * gn * 64,
                                 ns, st));
      for (const Fft16Step &s : p.interp) {
        if (s.kind == Fft16Step::kTransform) {
          RSB_TRY(run_transform(s));
          continue;
        }
        const uint64_t items = (uint64_t)ns * s.size * gn;
        const uint16_t *mc = s.cols == Fft16Program::kNoConst ? nullptr : d_cols + s.cols * 16;
        if (fft16_rt())
          fft16_mulxor_kernel<true><<<grid_for(items), kFft16Threads, 0, st>>>(
              buf[s.src_buf], regs_of[s.src_buf], s.src_start, buf[0], regs_of[0], s.dst_start, s.size, gn, ns, mc);
        else
          fft16_mulxor_kernel<false><<<grid_for(items), kFft16Threads, 0, st>>>(
              buf[s.src_buf], regs_of[s.src_buf], s.src_start, buf[0], regs_of[0], s.dst_start, s.size, gn, ns, mc);
        g_launches++;
        RSB_CU(cudaGetLastError());
      }
      for (const Fft16Eval &e : p.evals) {
        Fft16Step s{};
        s.kind = Fft16Step::kTransform;
        s.src_buf = 0;
        s.dst_buf = 2;
        s.size = t;
        s.cols = e.cols;
        RSB_TRY(run_transform(s));
        const uint32_t rows = e.r_hi - e.r_lo;
        fft16_store_kernel<<<grid_for((uint64_t)ns * rows * gn), kFft16Threads, 0, st>>>(
            buf[2] + (uint64_t)e.r_lo * gn * 16, t, rows, N, g0, gn, ns,
            d_ptrs ? nullptr : out_base + s0 * out_stripe + e.parity_row * out_row, out_row, out_stripe,
            d_ptrs ? d_ptrs + k + e.parity_row : nullptr);
        g_launches++;
        RSB_CU(cudaGetLastError());
      }
    }
  }
  return RS_OK;
}

}  // namespace rsb

extern "C" int rs_set_fft16_pass(int variant) {
  if (variant < 0 || variant > 2) return -1;
  const int old = rsb::fft16_pass_variant();
  rsb::fft16_pass_variant() = variant;
  return old;
}
