// Device arithmetic shared by the engine's kernels.
//
// Every rounding step is explicit (__fmaf_rn, __fdiv_rn, __fsqrt_rn, __fma_rn)
// and the kernels are compiled with -fmad=false, so the FP32 results do not
// depend on the compiler's contraction choices.
//
//   exp_m  : Cody-Waite reduction x = n ln2 + r (ln2 split in two parts) and the
//            degree-7 Taylor polynomial of e^r on |r| <= ln2/2, scaled by 2^n in
//            two exact power-of-two multiplications.
//   log_m  : x = m 2^e with m in [sqrt(1/2), sqrt(2)), log m = 2 atanh(s),
//            s = (m-1)/(m+1), odd series to s^11.
//   philox : Philox4x32-10 counter-based generator (Salmon, Moraes, Dror, Shaw,
//            "Parallel random numbers: as easy as 1, 2, 3", SC'11).
//   poisson: sequential-search inversion for lambda <= 10; larger lambda is split
//            into ceil(lambda/10) independent draws (a sum of independent Poisson
//            variables is Poisson); one Philox block gives the uniforms of four
//            consecutive time steps of an edge.
#pragma once
#include <cstdint>

namespace ngpu {

// Both functions compute the main path for every input and select the special results
// at the end (no branches).  rint(x log2 e) comes from the magic-number addition
// 1.5 * 2^23, which rounds to the nearest integer, ties to even, like rintf for
// |x log2 e| < 2^22; the scale 2^n is applied as 2^(n>>1) * 2^(n - (n>>1)), the first
// factor keeping the intermediate normal, so the result is the rounding of p * 2^n.
__device__ __forceinline__ float exp_m(float x) {
  // inputs outside [-103.97, 88.72] (and NaN) give meaningless bits on the main path, which
  // the selects at the end replace
  const float t = __fadd_rn(__fmul_rn(x, 1.44269502162933349609f), 12582912.0f);
  const float n = __fsub_rn(t, 12582912.0f);
  float r = __fmaf_rn(n, -0.693145751953125f, x);
  r = __fmaf_rn(n, -1.428606765330187045e-06f, r);
  float p = 1.98412701e-04f;
  p = __fmaf_rn(p, r, 1.38888892e-03f);
  p = __fmaf_rn(p, r, 8.33333377e-03f);
  p = __fmaf_rn(p, r, 4.16666679e-02f);
  p = __fmaf_rn(p, r, 1.66666672e-01f);
  p = __fmaf_rn(p, r, 0.5f);
  p = __fmaf_rn(p, r, 1.0f);
  p = __fmaf_rn(p, r, 1.0f);
  const int ni = (int)(__float_as_uint(t) - 0x4B400000u);
  const int n1 = ni >> 1;
  const int n2 = ni - n1;
  p = __fmul_rn(p, __uint_as_float((unsigned)(n1 + 127) << 23));
  p = __fmul_rn(p, __uint_as_float((unsigned)(n2 + 127) << 23));
  p = (x > 88.72283935546875f) ? __int_as_float(0x7f800000) : p;
  p = (x < -103.972084045410156f) ? 0.0f : p;
  return (x == x) ? p : x;
}

__device__ __forceinline__ float log_m(float x) {
  const bool sub = x < 1.17549435e-38f;
  const float xs = sub ? __fmul_rn(x, 16777216.0f) : x;
  const unsigned b = __float_as_uint(xs);
  int e = (int)((b >> 23) & 0xff) - (sub ? 151 : 127);
  float m = __uint_as_float((b & 0x7fffffu) | 0x3f800000u);
  const bool hi = m > 1.41421354f;
  m = hi ? __fmul_rn(m, 0.5f) : m;
  e += hi ? 1 : 0;
  const float s = __fdiv_rn(__fsub_rn(m, 1.0f), __fadd_rn(m, 1.0f));
  const float s2 = __fmul_rn(s, s);
  float q = 9.09090936e-02f;
  q = __fmaf_rn(q, s2, 1.11111112e-01f);
  q = __fmaf_rn(q, s2, 1.42857149e-01f);
  q = __fmaf_rn(q, s2, 2.00000003e-01f);
  q = __fmaf_rn(q, s2, 3.33333343e-01f);
  q = __fmaf_rn(q, s2, 1.0f);
  const float lm = __fmul_rn(__fmul_rn(2.0f, s), q);
  const float fe = (float)e;
  float res = __fmaf_rn(fe, 0.693145751953125f, __fmaf_rn(fe, 1.428606765330187045e-06f, lm));
  res = (x == __int_as_float(0x7f800000)) ? x : res;
  res = (x == 0.0f) ? __int_as_float(0xff800000) : res;
  return (x > 0.0f || x == 0.0f) ? res : __int_as_float(0x7fc00000);
}

struct U4 { uint32_t x, y, z, w; };

__device__ __forceinline__ U4 philox(U4 c, uint32_t k0, uint32_t k1) {
#pragma unroll
  for (int r = 0; r < 10; r++) {
    uint32_t lo0 = 0xD2511F53u * c.x, hi0 = __umulhi(0xD2511F53u, c.x);
    uint32_t lo1 = 0xCD9E8D57u * c.z, hi1 = __umulhi(0xCD9E8D57u, c.z);
    U4 n;
    n.x = hi1 ^ c.y ^ k0;
    n.y = lo1;
    n.z = hi0 ^ c.w ^ k1;
    n.w = lo0;
    c = n;
    k0 += 0x9E3779B9u;
    k1 += 0xBB67AE85u;
  }
  return c;
}

__device__ __forceinline__ float u01(uint32_t r) {
  return __fmul_rn(__fadd_rn((float)(r >> 8), 0.5f), 5.96046448e-08f);
}

// 1/k rounded to float, k = 0..64 (entry 0 unused): the inversion's recurrence
// multiplies by it instead of dividing.
#define NGPU_INV8(k) (float)(1.0 / (k)), (float)(1.0 / ((k) + 1)), (float)(1.0 / ((k) + 2)), \
    (float)(1.0 / ((k) + 3)), (float)(1.0 / ((k) + 4)), (float)(1.0 / ((k) + 5)), (float)(1.0 / ((k) + 6)), \
    (float)(1.0 / ((k) + 7))
static __constant__ float c_inv_k[65] = {0.0f, NGPU_INV8(1), NGPU_INV8(9), NGPU_INV8(17), NGPU_INV8(25),
                                         NGPU_INV8(33), NGPU_INV8(41), NGPU_INV8(49), NGPU_INV8(57)};
#undef NGPU_INV8

// Inversion by sequential search: the smallest k with u <= F(k), p(k) = p(k-1) lam / k
// starting from p(0) = emlam = exp(-lam).
__device__ __forceinline__ int poisson_small(float lam, float emlam, float u) {
  float p = emlam;
  float F = p;
  int k = 0;
  while (u > F && p > 9.31322575e-10f && k < 1000) {
    k++;
    const float ik = (k <= 64) ? c_inv_k[k] : __fdiv_rn(1.0f, (float)k);
    p = __fmul_rn(__fmul_rn(p, lam), ik);
    F = __fadd_rn(F, p);
  }
  return k;
}

__device__ __forceinline__ uint32_t word_of(const U4 &r, int w) {
  return w == 0 ? r.x : w == 1 ? r.y : w == 2 ? r.z : r.w;
}

// Philox block of direct edge `edge` for the four time indices 4*(tidx/4) .. +3 and
// chunk field j (0 for lam <= 10; 1.. for the chunks of a larger lam).
__device__ __forceinline__ U4 poisson_block(uint64_t seed, uint64_t edge, long long tidx, uint32_t j) {
  U4 c;
  c.x = (uint32_t)edge;
  c.y = (uint32_t)(edge >> 32);
  c.z = (uint32_t)((unsigned long long)tidx >> 2);
  c.w = ((uint32_t)((unsigned long long)tidx >> 34) & 0xffffu) | (j << 16);
  return philox(c, (uint32_t)seed ^ 0x6A09E667u, (uint32_t)(seed >> 32) ^ 0xBB67AE85u);
}

// n ~ Poisson(lam) of direct edge `edge` at time index `tidx`: word tidx % 4 of the edge's
// block for tidx / 4 (one Philox call serves four consecutive steps).
__device__ __forceinline__ int poisson_draw(float lam, uint64_t seed, uint64_t edge, long long tidx) {
  if (!(lam > 0.0f)) return 0;
  const int w = (int)(tidx & 3);
  if (lam <= 10.0f) return poisson_small(lam, exp_m(-lam), u01(word_of(poisson_block(seed, edge, tidx, 0), w)));
  const int m = (int)ceilf(__fdiv_rn(lam, 10.0f));
  const float lc = __fdiv_rn(lam, (float)m);
  const float emlc = exp_m(-lc);
  int n = 0;
  for (int j = 0; j < m; j++)
    n += poisson_small(lc, emlc, u01(word_of(poisson_block(seed, edge, tidx, (uint32_t)(j + 1)), w)));
  return n;
}

}  // namespace ngpu
