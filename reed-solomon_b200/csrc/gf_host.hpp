// Host-side field arithmetic and coefficient construction for the rs_b200 library.
//
// GF(2^8) is the field of the reference's src/galois.rs (x^8+x^4+x^3+x^2+1,
// generator 2); GF((2^8)^2) is its tower y^2 + y + 32 (src/galois16.rs:19-59), with
// elements packed (high << 8) | low.
//
// Generator and decode rows are built in closed form. The reference builds the
// systematic generator as vandermonde(n, k) * inverse(top k x k)
// (src/reedsolomon.rs:155-159, src/matrix.rs:183-196 with evaluation point r = r).
// That product maps the values of the unique degree < k polynomial at points
// 0..k-1 to its value at point r, so row r is the Lagrange basis on points 0..k-1
// evaluated at r. Likewise the reference's decode rows (inverse of the survivor rows,
// src/reedsolomon.rs:539-585, then generator rows for missing parity) compose to the
// Lagrange basis on the survivor points evaluated at each missing point. Linear maps
// are unique, so these rows are byte-identical to the reference's, at
// O(k^2 + rows * k) field operations instead of O(k^3).
#pragma once

#include <cstddef>
#include <cstdint>
#include <vector>

namespace rsb {

struct Gf8Tables {
  uint8_t log[256];
  uint8_t exp[512];
  Gf8Tables() {
    unsigned x = 1;
    for (unsigned i = 0; i < 255; i++) {
      exp[i] = (uint8_t)x;
      log[x] = (uint8_t)i;
      x <<= 1;
      if (x & 0x100) x ^= 0x11d;
    }
    for (unsigned i = 255; i < 512; i++) exp[i] = exp[i - 255];
    log[0] = 0;
  }
};

inline const Gf8Tables &gf8() {
  static const Gf8Tables t;
  return t;
}

inline uint8_t gf8_mul(uint8_t a, uint8_t b) {
  if (!a || !b) return 0;
  const Gf8Tables &t = gf8();
  return t.exp[t.log[a] + t.log[b]];
}

inline uint8_t gf8_inv(uint8_t a) {  // a != 0
  const Gf8Tables &t = gf8();
  return t.exp[255 - t.log[a]];
}

// Tower product (high*y + low)(high'*y + low') reduced by y^2 = y + 32.
inline uint16_t gf16_mul(uint16_t a, uint16_t b) {
  uint8_t ah = a >> 8, al = a & 0xff, bh = b >> 8, bl = b & 0xff;
  uint8_t p2 = gf8_mul(ah, bh);
  uint8_t p1 = gf8_mul(ah, bl) ^ gf8_mul(al, bh);
  uint8_t p0 = gf8_mul(al, bl);
  return (uint16_t)(((p1 ^ p2) << 8) | (uint8_t)(p0 ^ gf8_mul(p2, 32)));
}

// Inverse through the norm: the conjugate of high*y + low is high*y + (high + low)
// and their product lies in GF(2^8).
inline uint16_t gf16_inv(uint16_t a) {  // a != 0
  uint8_t ah = a >> 8, al = a & 0xff;
  uint16_t conj = (uint16_t)((ah << 8) | (uint8_t)(ah ^ al));
  uint8_t ni = gf8_inv((uint8_t)(gf16_mul(a, conj) & 0xff));
  return (uint16_t)((gf8_mul(conj >> 8, ni) << 8) | gf8_mul(conj & 0xff, ni));
}

// Multiplicative log/exp tables of GF((2^8)^2) for fast host construction; built
// from gf16_mul on first use with the smallest primitive element.
struct Gf16Tables {
  std::vector<uint16_t> log, exp;  // exp has 2*65535 entries
  Gf16Tables();
};
const Gf16Tables &gf16();

struct F8 {
  using T = uint8_t;
  static T mul(T a, T b) { return gf8_mul(a, b); }
  static T inv(T a) { return gf8_inv(a); }
  static T point(size_t i) { return (T)i; }
};

struct F16 {
  using T = uint16_t;
  static T mul(T a, T b) {
    if (!a || !b) return 0;
    const Gf16Tables &t = gf16();
    return t.exp[(size_t)t.log[a] + t.log[b]];
  }
  static T inv(T a) {
    const Gf16Tables &t = gf16();
    return t.exp[65535 - t.log[a]];
  }
  static T point(size_t i) { return (T)i; }
};

// rows[t][u] = L_u(point(targets[t])) where L_u is the Lagrange basis on the points
// of `nodes` (distinct indexes). A target equal to a node gives the unit row.
template <class F>
void lagrange_rows(const std::vector<size_t> &nodes, const std::vector<size_t> &targets,
                   std::vector<typename F::T> &rows) {
  using T = typename F::T;
  size_t k = nodes.size();
  rows.assign(targets.size() * k, 0);
  // Barycentric weights w_u = 1 / prod_{v != u} (x_u - x_v).
  std::vector<T> w(k);
  for (size_t u = 0; u < k; u++) {
    T prod = 1;
    T xu = F::point(nodes[u]);
    for (size_t v = 0; v < k; v++)
      if (v != u) prod = F::mul(prod, (T)(xu ^ F::point(nodes[v])));
    w[u] = F::inv(prod);
  }
  for (size_t t = 0; t < targets.size(); t++) {
    T xt = F::point(targets[t]);
    size_t hit = k;
    T ell = 1;  // prod_v (x_t - x_v)
    for (size_t v = 0; v < k; v++) {
      T d = (T)(xt ^ F::point(nodes[v]));
      if (d == 0) hit = v;
      ell = F::mul(ell, d);
    }
    T *row = &rows[t * k];
    if (hit < k) {
      row[hit] = 1;
      continue;
    }
    for (size_t u = 0; u < k; u++)
      row[u] = F::mul(F::mul(w[u], ell), F::inv((T)(xt ^ F::point(nodes[u]))));
  }
}

// Parity rows k..k+m-1 of the systematic generator (m x k, row-major).
template <class F>
void parity_rows(size_t k, size_t m, std::vector<typename F::T> &rows) {
  std::vector<size_t> nodes(k), targets(m);
  for (size_t i = 0; i < k; i++) nodes[i] = i;
  for (size_t j = 0; j < m; j++) targets[j] = k + j;
  lagrange_rows<F>(nodes, targets, rows);
}

}  // namespace rsb
