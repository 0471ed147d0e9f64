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
//            variables is Poisson).
#pragma once
#include <cstdint>

namespace ngpu {

__device__ __forceinline__ float exp_m(float x) {
  if (!(x == x)) return x;
  if (x > 88.72283935546875f) return __int_as_float(0x7f800000);
  if (x < -103.972084045410156f) return 0.0f;
  float n = rintf(__fmul_rn(x, 1.44269502162933349609f));
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
  int ni = (int)n;
  int n1 = ni / 2;
  int n2 = ni - n1;
  p = __fmul_rn(p, __int_as_float((n1 + 127) << 23));
  p = __fmul_rn(p, __int_as_float((n2 + 127) << 23));
  return p;
}

__device__ __forceinline__ float log_m(float x) {
  if (!(x > 0.0f)) return (x == 0.0f) ? __int_as_float(0xff800000) : __int_as_float(0x7fc00000);
  if (x == __int_as_float(0x7f800000)) return x;
  int e = 0;
  if (x < 1.17549435e-38f) { x = __fmul_rn(x, 16777216.0f); e = -24; }
  unsigned b = __float_as_uint(x);
  e += (int)((b >> 23) & 0xff) - 127;
  float m = __uint_as_float((b & 0x7fffffu) | 0x3f800000u);
  if (m > 1.41421354f) { m = __fmul_rn(m, 0.5f); e += 1; }
  float s = __fdiv_rn(__fsub_rn(m, 1.0f), __fadd_rn(m, 1.0f));
  float s2 = __fmul_rn(s, s);
  float q = 9.09090936e-02f;
  q = __fmaf_rn(q, s2, 1.11111112e-01f);
  q = __fmaf_rn(q, s2, 1.42857149e-01f);
  q = __fmaf_rn(q, s2, 2.00000003e-01f);
  q = __fmaf_rn(q, s2, 3.33333343e-01f);
  q = __fmaf_rn(q, s2, 1.0f);
  float lm = __fmul_rn(__fmul_rn(2.0f, s), q);
  float fe = (float)e;
  return __fmaf_rn(fe, 0.693145751953125f, __fmaf_rn(fe, 1.428606765330187045e-06f, lm));
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

__device__ __forceinline__ int poisson_small(float lam, float u) {
  float p = exp_m(-lam);
  float F = p;
  int k = 0;
  while (u > F && p > 9.31322575e-10f && k < 1000) {
    k++;
    p = __fdiv_rn(__fmul_rn(p, lam), (float)k);
    F = __fadd_rn(F, p);
  }
  return k;
}

// n ~ Poisson(lam) of direct edge `edge` at time index `tidx`.
__device__ __forceinline__ int poisson_draw(float lam, uint64_t seed, uint64_t edge, long long tidx) {
  if (!(lam > 0.0f)) return 0;
  int m = 1;
  float lc = lam;
  if (lam > 10.0f) {
    m = (int)ceilf(__fdiv_rn(lam, 10.0f));
    lc = __fdiv_rn(lam, (float)m);
  }
  uint32_t k0 = (uint32_t)seed ^ 0x6A09E667u;
  uint32_t k1 = (uint32_t)(seed >> 32) ^ 0xBB67AE85u;
  int n = 0;
  U4 r = {0, 0, 0, 0};
  for (int j = 0; j < m; j++) {
    if ((j & 3) == 0) {
      U4 c;
      c.x = (uint32_t)edge;
      c.y = (uint32_t)(edge >> 32);
      c.z = (uint32_t)tidx;
      c.w = ((uint32_t)((unsigned long long)tidx >> 32) & 0xffffu) | ((uint32_t)(j >> 2) << 16);
      r = philox(c, k0, k1);
    }
    uint32_t v = (j & 3) == 0 ? r.x : (j & 3) == 1 ? r.y : (j & 3) == 2 ? r.z : r.w;
    n += poisson_small(lc, u01(v));
  }
  return n;
}

}  // namespace ngpu
