// f32x2.cuh — two lattice cells per instruction: the D3Q19 moments and BGK / TRT
// collision (with Guo forcing) on packed pairs of FP32 values.
//
// sm_100 executes FP32 add, subtract, multiply and fused multiply-add on a pair of
// values held in one 64-bit register pair (PTX add/sub/mul/fma .f32x2).  The kernels
// that update two or four x-adjacent cells per thread keep each population of the two
// cells as one such pair (cell 0 in the low lane, cell 1 in the high lane), so every
// arithmetic instruction of the collision serves both cells: the step kernels of this
// path are bound by instruction issue, not by the FP32 pipe.  Each lane is rounded
// exactly as the scalar FP32 operation (round to nearest even); the expressions follow
// the scalar collide() / moments() of aa_impl.cuh operation for operation, with the
// multiply-adds written out as fma.
#pragma once
#include <cuda_fp16.h>
#include <stdint.h>

#include "lbm_internal.cuh"

namespace lbm {

struct F2 {
  unsigned long long v;
};

__device__ __forceinline__ F2 f2(float lo, float hi) {
  F2 r;
  asm("mov.b64 %0, {%1, %2};" : "=l"(r.v) : "f"(lo), "f"(hi));
  return r;
}
__device__ __forceinline__ F2 f2s(float a) { return f2(a, a); }
__device__ __forceinline__ void f2split(F2 x, float& lo, float& hi) {
  asm("mov.b64 {%0, %1}, %2;" : "=f"(lo), "=f"(hi) : "l"(x.v));
}
__device__ __forceinline__ float f2lo(F2 x) {
  float a, b;
  f2split(x, a, b);
  return a;
}
__device__ __forceinline__ float f2hi(F2 x) {
  float a, b;
  f2split(x, a, b);
  return b;
}
__device__ __forceinline__ F2 add(F2 a, F2 b) {
  F2 d;
  asm("add.rn.f32x2 %0, %1, %2;" : "=l"(d.v) : "l"(a.v), "l"(b.v));
  return d;
}
__device__ __forceinline__ F2 sub(F2 a, F2 b) {
  F2 d;
  asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(d.v) : "l"(a.v), "l"(b.v));
  return d;
}
__device__ __forceinline__ F2 mul(F2 a, F2 b) {
  F2 d;
  asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(d.v) : "l"(a.v), "l"(b.v));
  return d;
}
// a * b + c with one rounding per lane
__device__ __forceinline__ F2 fma(F2 a, F2 b, F2 c) {
  F2 d;
  asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(d.v) : "l"(a.v), "l"(b.v), "l"(c.v));
  return d;
}
// per-lane 1/x (one MUFU instruction per lane; ~1 ulp, as the scalar recip())
__device__ __forceinline__ F2 rcp(F2 x) {
  float a, b;
  f2split(x, a, b);
  asm("rcp.approx.ftz.f32 %0, %0;" : "+f"(a));
  asm("rcp.approx.ftz.f32 %0, %0;" : "+f"(b));
  return f2(a, b);
}
// half2 <-> pair of FP32 (the low half is the low lane)
__device__ __forceinline__ F2 f2_from_half2(uint32_t h) {
  const __half2 v = *reinterpret_cast<const __half2*>(&h);
  return f2(__low2float(v), __high2float(v));
}
__device__ __forceinline__ uint32_t half2_from_f2(F2 x) {
  float a, b;
  f2split(x, a, b);
  const __half2 v = __floats2half2_rn(a, b);
  return *reinterpret_cast<const uint32_t*>(&v);
}
// lane select: lane k of the result is lane k of b where bit k of `m` is set, else of a
__device__ __forceinline__ F2 f2sel(F2 a, F2 b, bool take_lo, bool take_hi) {
  float a0, a1, b0, b1;
  f2split(a, a0, a1);
  f2split(b, b0, b1);
  return f2(take_lo ? b0 : a0, take_hi ? b1 : a1);
}

// c_d . v for the even directions d = 2q (their opposites d + 1 carry the negated value):
// (1,0,0) (0,1,0) (0,0,1) (1,1,0) (1,0,1) (0,1,1) (1,-1,0) (1,0,-1) (0,1,-1)
__device__ __forceinline__ F2 cdot_even(int q, F2 x, F2 y, F2 z) {
  switch (q) {
    case 0: return x;
    case 1: return y;
    case 2: return z;
    case 3: return add(x, y);
    case 4: return add(x, z);
    case 5: return add(y, z);
    case 6: return sub(x, y);
    case 7: return sub(x, z);
    default: return sub(y, z);
  }
}

// Relaxation rates and body acceleration of a step, as uniform scalars.
struct Coll2 {
  float om_p, om_m;
  float gx, gy, gz;
};

// rho and the velocity (with the Guo half-force shift) of two cells; DEV: f holds the
// deviations g = f - w rho0 (rho = rho0 + sum g, j = sum c g).  Mirrors moments().
template <int FORCE, bool DEV>
__device__ __forceinline__ void moments2(const F2* f, const Coll2& k, const float rho0, F2& rho, F2& ux, F2& uy,
                                         F2& uz) {
  F2 sp[9], tp[9];
#pragma unroll
  for (int q = 0; q < 9; q++) {
    sp[q] = add(f[2 * q], f[2 * q + 1]);
    tp[q] = sub(f[2 * q], f[2 * q + 1]);
  }
  F2 r = add(add(add(sp[0], sp[1]), add(sp[2], sp[3])), add(add(sp[4], sp[5]), add(sp[6], sp[7])));
  r = add(r, add(sp[8], f[18]));
  // j = sum over the even directions of c_d (f_d - f_d+1)
  const F2 jx = add(add(add(tp[0], tp[3]), add(tp[4], tp[6])), tp[7]);
  const F2 jy = add(sub(add(tp[1], tp[3]), tp[6]), add(tp[5], tp[8]));
  const F2 jz = sub(sub(add(add(tp[2], tp[4]), tp[5]), tp[7]), tp[8]);
  if (DEV) r = add(r, f2s(rho0));
  const F2 inv = rcp(r);
  rho = r;
  if (FORCE) {
    ux = fma(jx, inv, f2s(0.5f * k.gx));
    if (FORCE != 2) {
      uy = fma(jy, inv, f2s(0.5f * k.gy));
      uz = fma(jz, inv, f2s(0.5f * k.gz));
    } else {
      uy = mul(jy, inv);
      uz = mul(jz, inv);
    }
  } else {
    ux = mul(jx, inv);
    uy = mul(jy, inv);
    uz = mul(jz, inv);
  }
}

// BGK / TRT with Guo forcing for two cells; the post-collision value of direction d is
// handed to emit(d, value) as soon as it is known (pairs (d, d+1) in turn, then the rest
// direction), so a caller can store it at once and the 19 results never need to be live
// together.  DEV: f and the results are deviations g = f - w rho0.  Mirrors collide().
template <bool TRT, int FORCE, bool DEV, class Emit>
__device__ __forceinline__ void collide2(const F2* f, const Coll2& k, const float rho0, const F2 rho, const F2 ux,
                                         const F2 uy, const F2 uz, Emit&& emit) {
  constexpr float W1 = 1.0f / 18.0f, W2 = 1.0f / 36.0f, W0 = 1.0f / 3.0f;
  const F2 usq = fma(ux, ux, fma(uy, uy, mul(uz, uz)));
  const F2 base = fma(f2s(-1.5f), usq, f2s(1.0f));
  F2 Fx = f2s(0.f), Fy = f2s(0.f), Fz = f2s(0.f), m3uF = f2s(0.f);
  if (FORCE == 2) {
    Fx = mul(rho, f2s(k.gx));
    m3uF = mul(f2s(-3.0f), mul(ux, Fx));
  } else if (FORCE) {
    Fx = mul(rho, f2s(k.gx));
    Fy = mul(rho, f2s(k.gy));
    Fz = mul(rho, f2s(k.gz));
    m3uF = mul(f2s(-3.0f), fma(ux, Fx, fma(uy, Fy, mul(uz, Fz))));
  }
  if (!TRT) {
    const float om = k.om_p, omc = 1.0f - k.om_p;
    const float fac = 1.0f - 0.5f * om;
    const float G1 = fac * W1, G2 = fac * W2;
    // omega * e = B + T (c.u)^2 ; omega * o = O (c.u)
    F2 B1, B2;
    if (DEV) {
      const F2 rb = fma(rho, base, f2s(-rho0));
      B1 = mul(f2s(om * W1), rb);
      B2 = mul(f2s(om * W2), rb);
      if (FORCE) {  // the direction-independent source part joins the constant
        B1 = fma(f2s(G1), m3uF, B1);
        B2 = fma(f2s(G2), m3uF, B2);
      }
    } else {
      const F2 rbase = mul(rho, base);
      B1 = mul(f2s(om * W1), rbase);
      B2 = mul(f2s(om * W2), rbase);
    }
    const F2 T1 = mul(f2s(4.5f * om * W1), rho), T2 = mul(f2s(4.5f * om * W2), rho);
    const F2 O1 = mul(f2s(3.0f * om * W1), rho), O2 = mul(f2s(3.0f * om * W2), rho);
    const F2 OMC = f2s(omc);
#pragma unroll
    for (int q = 0; q < 9; q++) {
      const int d = 2 * q;
      const bool c1 = d < 6;
      const F2 cu = cdot_even(q, ux, uy, uz);
      F2 e = fma(c1 ? T1 : T2, mul(cu, cu), c1 ? B1 : B2);
      F2 o = mul(c1 ? O1 : O2, cu);
      if (FORCE) {
        const float G = c1 ? G1 : G2;
        if (FORCE == 2 && cx(d) == 0) {  // c.F = 0
          if (!DEV) e = fma(f2s(G), m3uF, e);
        } else {
          const F2 cF = FORCE == 2 ? Fx : cdot_even(q, Fx, Fy, Fz);  // even directions: c_x >= 0
          if (DEV)
            e = fma(f2s(9.0f * G), mul(cu, cF), e);
          else
            e = fma(f2s(G), fma(f2s(9.0f), mul(cu, cF), m3uF), e);
          o = fma(f2s(3.0f * G), cF, o);
        }
      }
      emit(d, fma(OMC, f[d], add(e, o)));
      emit(d + 1, fma(OMC, f[d + 1], sub(e, o)));
    }
    F2 e0 = DEV ? mul(f2s(om * W0), fma(rho, base, f2s(-rho0))) : mul(f2s(om * W0), mul(rho, base));
    if (FORCE) e0 = fma(f2s(fac * W0), m3uF, e0);
    emit(18, fma(OMC, f[18], e0));
  } else {
    const float hp = 0.5f * k.om_p, hm = 0.5f * k.om_m;
    const float fac_p = 1.0f - hp, fac_m = 1.0f - hm;
    const F2 HP = f2s(hp), HM = f2s(hm), OMP = f2s(-k.om_p), OMM = f2s(-k.om_m);
#pragma unroll
    for (int q = 0; q < 9; q++) {
      const int d = 2 * q;
      const float w = d < 6 ? W1 : W2;
      const F2 cu = cdot_even(q, ux, uy, uz);
      const F2 be = fma(f2s(4.5f), mul(cu, cu), base);
      const F2 e = DEV ? mul(f2s(w), fma(rho, be, f2s(-rho0))) : mul(mul(rho, f2s(w)), be);
      const F2 o = mul(mul(f2s(3.0f * w), rho), cu);
      // A = om_p (f+ - e), Bm = om_m (f- - o), f+- = (f_d +- f_d+1)/2
      F2 A = fma(HP, add(f[d], f[d + 1]), mul(OMP, e));
      F2 Bm = fma(HM, sub(f[d], f[d + 1]), mul(OMM, o));
      if (FORCE) {
        if (FORCE == 2 && cx(d) == 0) {  // c.F = 0
          A = fma(f2s(-fac_p * w), m3uF, A);
        } else {
          const F2 cF = FORCE == 2 ? Fx : cdot_even(q, Fx, Fy, Fz);
          A = fma(f2s(-fac_p * w), fma(f2s(9.0f), mul(cu, cF), m3uF), A);
          Bm = fma(f2s(-fac_m * 3.0f * w), cF, Bm);
        }
      }
      emit(d, sub(sub(f[d], A), Bm));
      emit(d + 1, add(sub(f[d + 1], A), Bm));
    }
    const F2 e0 = DEV ? mul(f2s(W0), fma(rho, base, f2s(-rho0))) : mul(mul(rho, f2s(W0)), base);
    F2 v = fma(OMP, sub(f[18], e0), f[18]);
    if (FORCE) v = fma(f2s(fac_p * W0), m3uF, v);
    emit(18, v);
  }
}

}  // namespace lbm
