// Offline search for the bitsliced FFT encode's subspace basis (kernels_fft.cuh, fftc::kBasis).
//
// The (K, K) encode evaluates, on the parity points {K .. 2K-1}, the polynomial of degree < K
// through the data points {0 .. K-1}. Those values do not depend on how the additive FFT
// enumerates the subspace V = {0 .. K-1}: any ordered basis v_0 .. v_{n-1} of V (register i
// holds point P(i) = XOR of v_j over the bits j of i) and any representative beta of the coset
// K + V (output register i holds point beta ^ P(i)) give the same parity bytes, only in another
// register order. The butterfly constants, and so the XOR networks of the constant multiplies,
// do change with the choice. This program scores every admissible (basis, beta) with the
// kernel's per-lane LOP3 count and prints the cheapest.
//
// Admissible: with lane groups of 2^W lanes the low W register bits are lane bits; v_0 ..
// v_{W-1} must be single bits and the other vectors clear of them, so that a lane's shard index
// stays (compile-time part) + (per-lane part).
//
// Cost per lane (LOP3 count of the compiled XOR networks; register XORs are the same for every
// choice and left out): local levels L >= W hold K/2^(W+1) butterflies per lane, the inverse
// costing mul(C) and the forward min(mul(C), mul(C ^ 1)) (it may compute hi' = lo ^ (C^1) hi and
// lo' = hi' ^ hi instead); cross-lane levels L < W cost, per slot, the block constant's multiply
// plus, for every lane bit T in (L, W), a masked multiply by WHAT_L(v_T).
//
// Build and run: gcc -O2 -o fft_basis_search fft_basis_search.c && ./fft_basis_search
#include <stdint.h>
#include <stdio.h>
#include <string.h>

static uint8_t LOG[256], EXP[512];
static int cost_acc[256], cost_set[256];

static uint8_t gm(uint8_t a, uint8_t b) { return (a && b) ? EXP[LOG[a] + LOG[b]] : 0; }
static uint8_t ginv(uint8_t a) { return EXP[255 - LOG[a]]; }

static void init_tables(void) {
  int x = 1;
  for (int i = 0; i < 255; i++) {
    EXP[i] = EXP[i + 255] = (uint8_t)x;
    LOG[x] = (uint8_t)i;
    x <<= 1;
    if (x & 256) x ^= 0x11d;
  }
  for (int c = 0; c < 256; c++) {
    int acc = 0, set = 0;
    for (int b = 0; b < 8; b++) {
      int nb = 0;
      for (int bp = 0; bp < 8; bp++) nb += (gm((uint8_t)c, (uint8_t)(1 << bp)) >> b) & 1;
      acc += (nb + 1) / 2;           // d ^= XOR of nb planes
      set += nb > 1 ? nb / 2 : 0;    // d = XOR of nb planes
    }
    cost_acc[c] = c == 0 ? 0 : c == 1 ? 8 : acc;
    cost_set[c] = c == 0 ? 0 : set;
  }
}

// Normalised subspace polynomials of the basis, on the points 0 .. 2K-1.
static void what_tables(int n, const uint8_t *v, uint8_t W[8][256]) {
  const int K = 1 << n;
  uint8_t raw[8][256];
  for (int y = 0; y < 2 * K; y++) raw[0][y] = (uint8_t)y;
  for (int l = 0; l + 1 < n; l++)
    for (int y = 0; y < 2 * K; y++) raw[l + 1][y] = gm(raw[l][y], raw[l][y] ^ raw[l][v[l]]);
  for (int l = 0; l < n; l++) {
    const uint8_t iv = ginv(raw[l][v[l]]);
    for (int y = 0; y < 2 * K; y++) W[l][y] = gm(raw[l][y], iv);
  }
}

static long score(int n, int w, const uint8_t *v, int beta, uint8_t W[8][256], const uint8_t *P) {
  const int K = 1 << n, S = K >> w;
  long c = 0;
  for (int inv = 1; inv >= 0; inv--) {
    const int b = inv ? 0 : beta;
    for (int l = 0; l < n; l++) {
      if (l >= w) {
        for (int base = 0; base < K; base += 2 << l) {
          const uint8_t C = W[l][b ^ P[base]];
          int k = cost_acc[C];
          if (!inv && C != 0 && cost_acc[C ^ 1] < k) k = cost_acc[C ^ 1];
          c += (long)(1 << (l - w)) * k;  // the block's butterflies held by one lane
        }
      } else {
        for (int j = 0; j < S; j++) {
          const uint8_t C = W[l][b ^ P[j << w]];
          c += inv ? cost_acc[C] : cost_set[C];
          for (int t = l + 1; t < w; t++) c += cost_set[W[l][v[t]]] + 8;
        }
      }
    }
  }
  return c;
}

// K = 128 has too many bases to enumerate: a seeded sample of admissible bases instead.
static void sample(int n, int w, long samples) {
  const int K = 1 << n;
  uint64_t st = 0x9e3779b97f4a7c15ull;
  long best = -1;
  uint8_t best_v[8] = {0};
  int best_beta = 0;
  for (long it = 0; it < samples; it++) {
    uint8_t v[8], span[128] = {1};
    int lanes = 0, d = 0;
    while (d < n) {
      st ^= st << 13, st ^= st >> 7, st ^= st << 17;
      const int c = (int)(st % (uint64_t)K);
      if (c == 0 || span[c]) continue;
      if (d < w ? (c & (c - 1)) != 0 : (c & lanes) != 0) continue;
      if (d < w) lanes |= c;
      v[d++] = (uint8_t)c;
      for (int y = 0; y < K; y++)
        if (span[y]) span[y ^ c] = 1;
    }
    uint8_t W[8][256], P[128];
    what_tables(n, v, W);
    for (int i = 0; i < K; i++) {
      uint8_t p = 0;
      for (int j = 0; j < n; j++)
        if ((i >> j) & 1) p ^= v[j];
      P[i] = p;
    }
    for (int beta = K; beta < 2 * K; beta++) {
      const long s = score(n, w, v, beta, W, P);
      if (best < 0 || s < best) {
        best = s;
        memcpy(best_v, v, 8);
        best_beta = beta;
      }
    }
  }
  uint8_t W[8][256], P[128], v[8] = {1, 2, 4, 8, 16, 32, 64, 128};
  what_tables(n, v, W);
  for (int i = 0; i < K; i++) P[i] = (uint8_t)i;
  printf("K=%3d W=%d standard=%5ld best=%5ld  {{", K, w, score(n, w, v, K, W, P), best);
  for (int j = 0; j < 8; j++) printf("%d%s", j < n ? best_v[j] : 0, j < 7 ? ", " : "");
  printf("}, %d}  (sampled)\n", best_beta);
}

static void search(int n, int w) {
  const int K = 1 << n;
  long best = -1, std_cost = -1;
  uint8_t best_v[8] = {0};
  int best_beta = 0;
  // Enumerate ordered bases depth-first.
  uint8_t v[8];
  int cand[8] = {0};
  uint8_t in_span[9][128];
  memset(in_span, 0, sizeof in_span);
  in_span[0][0] = 1;
  int depth = 0;
  cand[0] = 0;
  while (depth >= 0) {
    const int c = ++cand[depth];
    if (c >= K) {
      cand[depth] = 0;
      depth--;
      continue;
    }
    if (in_span[depth][c]) continue;
    if (depth < w && (c & (c - 1))) continue;
    if (depth >= w) {
      int bad = 0;
      for (int d = 0; d < w; d++) bad |= (c & v[d]) != 0;
      if (bad) continue;
    }
    v[depth] = (uint8_t)c;
    for (int y = 0; y < K; y++) in_span[depth + 1][y] = in_span[depth][y] | in_span[depth][y ^ c];
    if (depth + 1 < n) {
      depth++;
      cand[depth] = 0;
      continue;
    }
    uint8_t W[8][256], P[128];
    what_tables(n, v, W);
    for (int i = 0; i < K; i++) {
      uint8_t p = 0;
      for (int j = 0; j < n; j++)
        if ((i >> j) & 1) p ^= v[j];
      P[i] = p;
    }
    int is_std = 1;
    for (int j = 0; j < n; j++) is_std &= v[j] == (1 << j);
    for (int beta = K; beta < 2 * K; beta++) {
      const long s = score(n, w, v, beta, W, P);
      if (is_std && beta == K) std_cost = s;
      if (best < 0 || s < best) {
        best = s;
        memcpy(best_v, v, 8);
        best_beta = beta;
      }
    }
  }
  printf("K=%3d W=%d standard=%5ld best=%5ld  {{", K, w, std_cost, best);
  for (int j = 0; j < 8; j++) printf("%d%s", j < n ? best_v[j] : 0, j < 7 ? ", " : "");
  printf("}, %d}\n", best_beta);
}

int main(void) {
  init_tables();
  const int cases[][2] = {{1, 1}, {2, 1}, {3, 1}, {4, 1}, {4, 2}, {5, 1}, {5, 2}, {6, 2}, {6, 3}};
  for (unsigned i = 0; i < sizeof cases / sizeof cases[0]; i++) search(cases[i][0], cases[i][1]);
  sample(7, 3, 20000);
  sample(7, 4, 20000);
  return 0;
}
