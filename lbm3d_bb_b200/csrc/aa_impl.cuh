// aa_impl.cuh — configurable D3Q19 step as one fused AA-pattern kernel (device code
// and launch templates).  Each storage precision is instantiated in its own
// translation unit (kernels_aa_fp32.cu, kernels_aa_fp64.cu, kernels_aa_fp16.cu).
//
// One population array A (SoA: A[d*plane + node]) is updated in place.  Steps
// alternate between two phases:
//   even phase: node x reads S[d,x] = A[d][x], collides, and writes its
//               post-collision f*[dbar] into A[d][x] (swapped slots);
//   odd phase:  node x pulls S[d,x] = A[dbar][x - c_d], collides, and pushes
//               f*[d] into A[d][x + c_d].
// Every slot is read and written by exactly one thread per phase, so the kernel
// is race-free and moves 2 * 19 populations per node per step.
//
// Boundaries are "own-slot" rules: when the source x - c_d of an incoming
// population lies outside a non-periodic face or in a solid node, the value is a
// function of node x alone (bounce-back, equilibrium, zero-gradient) and is kept
// in A[d][x], a slot no other node touches in either phase.  This covers
// SolidBC.jl's moving-wall bounce-back (SBB!_gpu, SolidBC.jl:160-210) and the
// face conditions of OtherBC.jl (velocity_BC!_gpu, OtherBC.jl:112-169) in the
// configurable form.  Links are resolved from the node flag bytes (no CSR on the
// hot path); the momentum exchange of MEA.jl:76-116 is accumulated in FP64 and
// reduced with warp shuffles, one atomic per block and component.
//
// Moving bodies: the flags of the previous step decide which incoming slots hold
// boundary values (read side), the current flags decide what is written; nodes
// uncovered by the body are refilled with the equilibrium at the body velocity.
// A fresh node's emitted populations toward old fluid neighbours are recomputed by
// those neighbours (same __noinline__ routine, bit-identical), which keeps the odd
// phase race-free.
#pragma once
#include "lbm_internal.cuh"
#include "lbm_kernels.h"

#ifndef LBM_MINB_F32
#define LBM_MINB_F32 4
#endif
#ifndef LBM_MINB_F16
#define LBM_MINB_F16 4
#endif

// blocks of BATCH_ITEM threads per SM that the batched kernel's register budget allows:
// FP32 6 (80 registers; 2 % faster than 8 on the 512-domain sweep, 4 was slower), the
// other storages 2 x MIN_BLOCKS
#ifndef LBM_BATCH_MINB
#define LBM_BATCH_MINB(SP) (sizeof(typename SP::S) == 4 ? 6 : 2 * SP::MIN_BLOCKS)
#endif

namespace lbm {

// ---- storage policies ------------------------------------------------------------
// ld/st convert between the stored value and the population f; ld_raw/st_raw move
// the stored value as it is.  DEV: the stored value is the deviation g = f - w_d rho0,
// and the fast path computes in deviations (no conversion per population).
struct StF32 {
  using S = float;
  using C = float;
  static constexpr int MIN_BLOCKS = LBM_MINB_F32;  // 256 x 4 threads -> at most 64 registers
  static constexpr bool DEV = false;
  static __device__ __forceinline__ C ld(const S* p, int, C) { return *p; }
  static __device__ __forceinline__ void st(S* p, C v, int, C) { *p = v; }
  static __device__ __forceinline__ C ld_raw(const S* p) { return *p; }
  static __device__ __forceinline__ void st_raw(S* p, C v) { *p = v; }
};
struct StF64 {
  using S = double;
  using C = double;
  static constexpr int MIN_BLOCKS = 2;
  static constexpr bool DEV = false;
  static __device__ __forceinline__ C ld(const S* p, int, C) { return *p; }
  static __device__ __forceinline__ void st(S* p, C v, int, C) { *p = v; }
  static __device__ __forceinline__ C ld_raw(const S* p) { return *p; }
  static __device__ __forceinline__ void st_raw(S* p, C v) { *p = v; }
};
// FP16 deviation from the rest equilibrium: stored h = f - w_d*rho0, computed in FP32.
struct StF16 {
  using S = __half;
  using C = float;
  static constexpr int MIN_BLOCKS = LBM_MINB_F16;
  static constexpr bool DEV = true;
  static __device__ __forceinline__ C ld(const S* p, int d, C rho0) {
    return wgt<float>(d) * rho0 + __half2float(*p);
  }
  static __device__ __forceinline__ void st(S* p, C v, int d, C rho0) {
    *p = __float2half_rn(v - wgt<float>(d) * rho0);
  }
  static __device__ __forceinline__ C ld_raw(const S* p) { return __half2float(*p); }
  static __device__ __forceinline__ void st_raw(S* p, C v) { *p = __float2half_rn(v); }
};

// Storage policy with explicit global-space population accesses (ld.global.cg and
// st.global.cg): the batched kernel takes each domain's population pointer from a device
// table, so the compiler cannot infer the address space and would emit generic loads and
// stores.  Same values as the wrapped policy.
template <class Base>
struct GlobalSpace : Base {
  using S = typename Base::S;
  using C = typename Base::C;
  static __device__ __forceinline__ C ld(const S* p, int d, C rho0) {
    const S v = __ldcg(p);
    return Base::ld(&v, d, rho0);
  }
  static __device__ __forceinline__ void st(S* p, C v, int d, C rho0) {
    S t;
    Base::st(&t, v, d, rho0);
    __stcg(p, t);
  }
  static __device__ __forceinline__ C ld_raw(const S* p) {
    const S v = __ldcg(p);
    return Base::ld_raw(&v);
  }
  static __device__ __forceinline__ void st_raw(S* p, C v) {
    S t;
    Base::st_raw(&t, v);
    __stcg(p, t);
  }
};

// ---- collision ---------------------------------------------------------------------
template <class C>
struct Coll {
  C om_p, om_m;  // relaxation rates
  C gx, gy, gz;  // body acceleration
};

// 1/rho: one MUFU instruction in FP32 (rho is O(1), the ~1 ulp error is far below
// the storage precision); exact division in FP64.
__device__ __forceinline__ float recip(float r) {
  float y;
  asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(r));
  return y;
}
__device__ __forceinline__ double recip(double r) { return 1.0 / r; }

// Moments from the nine opposite-direction pairs (d, d+1): s = f_d + f_{d+1},
// t = f_d - f_{d+1}; rho = sum s + f_18, j = sum over pairs of c_d t.  Then
// u = j/rho + g/2 (Guo).
// DEV: f holds deviations g = f - w rho0 (sum w = 1, sum w c = 0: rho = rho0 + sum g,
// j = sum c g).
template <class C, int FORCE, bool DEV = false>
__device__ __forceinline__ void moments(const C* f, const Coll<C>& k, C& rho, C& ux, C& uy, C& uz,
                                        const C rho0 = C(0)) {
  C sp[9], tp[9];
#pragma unroll
  for (int q = 0; q < 9; q++) {
    sp[q] = f[2 * q] + f[2 * q + 1];
    tp[q] = f[2 * q] - f[2 * q + 1];
  }
  C r = ((sp[0] + sp[1]) + (sp[2] + sp[3])) + ((sp[4] + sp[5]) + (sp[6] + sp[7])) + (sp[8] + f[18]);
  C jx = C(0), jy = C(0), jz = C(0);
#pragma unroll
  for (int q = 0; q < 9; q++) {
    const int d = 2 * q;
    if (cx(d) == 1) jx += tp[q];
    if (cx(d) == -1) jx -= tp[q];
    if (cy(d) == 1) jy += tp[q];
    if (cy(d) == -1) jy -= tp[q];
    if (cz(d) == 1) jz += tp[q];
    if (cz(d) == -1) jz -= tp[q];
  }
  if (DEV) r += rho0;
  const C inv = recip(r);
  rho = r;
  ux = jx * inv;
  uy = jy * inv;
  uz = jz * inv;
  if (FORCE) {
    ux += C(0.5) * k.gx;
    if (FORCE != 2) {  // FORCE == 2: acceleration along x only
      uy += C(0.5) * k.gy;
      uz += C(0.5) * k.gz;
    }
  }
}

template <class C>
__device__ __forceinline__ C cdot(int d, C ux, C uy, C uz) {
  C s = C(0);
  if (cx(d) == 1) s += ux;
  if (cx(d) == -1) s -= ux;
  if (cy(d) == 1) s += uy;
  if (cy(d) == -1) s -= uy;
  if (cz(d) == 1) s += uz;
  if (cz(d) == -1) s -= uz;
  return s;
}

template <class C>
__device__ __forceinline__ C feq(int d, C rho, C ux, C uy, C uz) {
  C cu = cdot<C>(d, ux, uy, uz);
  C usq = ux * ux + uy * uy + uz * uz;
  return wgt<C>(d) * rho * (C(1) + C(3) * cu + C(4.5) * cu * cu - C(1.5) * usq);
}

// BGK / TRT with Guo forcing, f -> p, written per opposite pair (d, d+1) with
// c_{d+1} = -c_d: the equilibrium splits into an even part
// e = w rho (1 - 1.5 u^2 + 4.5 (c.u)^2) and an odd part o = 3 w rho (c.u), the Guo
// source S_d = w [3 (c_d - u).F + 9 (c_d.u)(c_d.F)] into w (9 (c.u)(c.F) - 3 u.F) and
// 3 w (c.F).  Relaxation rates and weights are folded per weight class.
// DEV: f and p are deviations g = f - w rho0.  Only the even equilibrium part carries
// the offset: e - w rho0 = w (rho (1 - 1.5 u^2 + 4.5 (c.u)^2) - rho0); in the TRT form the
// offsets of f+ and of e cancel because hp = om_p / 2.
template <class C, bool TRT, int FORCE, bool DEV = false>
__device__ __forceinline__ void collide(const C* f, C* p, const Coll<C>& k, C rho, C ux, C uy, C uz,
                                        const C rho0 = C(0)) {
  const C usq = ux * ux + uy * uy + uz * uz;
  const C base = C(1) - C(1.5) * usq;
  C Fx = C(0), Fy = C(0), Fz = C(0), m3uF = C(0);
  if (FORCE == 2) {  // acceleration along x only: the y and z terms are exact zeros
    Fx = rho * k.gx;
    m3uF = C(-3) * (ux * Fx);
  } else if (FORCE) {
    Fx = rho * k.gx;
    Fy = rho * k.gy;
    Fz = rho * k.gz;
    m3uF = C(-3) * (ux * Fx + uy * Fy + uz * Fz);
  }
  const C wr1 = rho * wgt<C>(0), wr2 = rho * wgt<C>(6), wr0 = rho * wgt<C>(18);
  if (!TRT) {
    const C om = k.om_p, omc = C(1) - k.om_p;
    // omega * e = B + T (c.u)^2 ; omega * o = O (c.u)
    const C rb = rho * base - rho0;  // DEV only
    C B1 = DEV ? om * wgt<C>(0) * rb : om * wr1 * base, B2 = DEV ? om * wgt<C>(6) * rb : om * wr2 * base;
    const C T1 = C(4.5) * om * wr1, T2 = C(4.5) * om * wr2;
    const C O1 = C(3) * om * wr1, O2 = C(3) * om * wr2;
    const C fac = C(1) - C(0.5) * om;
    const C G1 = fac * wgt<C>(0), G2 = fac * wgt<C>(6);
    // FP16 deviations: the direction-independent source part w (-3 u.F) joins the
    // constant of e (one FMA less per direction pair; measured faster on B200 for the
    // issue-bound FP16 kernels, slower for FP32, which keeps the unfolded form)
    if (FORCE && DEV) {
      B1 += G1 * m3uF;
      B2 += G2 * m3uF;
    }
#pragma unroll
    for (int q = 0; q < 9; q++) {
      const int d = 2 * q;
      const bool c1 = d < 6;
      const C cu = cdot<C>(d, ux, uy, uz);
      C e = (c1 ? T1 : T2) * (cu * cu) + (c1 ? B1 : B2);
      C o = (c1 ? O1 : O2) * cu;
      if (FORCE) {
        const C G = c1 ? G1 : G2;
        if (FORCE == 2 && cx(d) == 0) {  // c.F = 0
          if (!DEV) e += G * m3uF;
        } else {
          const C cF = FORCE == 2 ? (cx(d) > 0 ? Fx : -Fx) : cdot<C>(d, Fx, Fy, Fz);
          if (DEV)
            e += (C(9) * G) * (cu * cF);
          else
            e += G * (C(9) * (cu * cF) + m3uF);
          o += (C(3) * G) * cF;
        }
      }
      p[d] = omc * f[d] + (e + o);
      p[d + 1] = omc * f[d + 1] + (e - o);
    }
    C e0 = DEV ? om * wgt<C>(18) * rb : om * wr0 * base;
    if (FORCE) e0 += fac * wgt<C>(18) * m3uF;
    p[18] = omc * f[18] + e0;
  } else {
    const C hp = C(0.5) * k.om_p, hm = C(0.5) * k.om_m;
    const C fac_p = C(1) - hp, fac_m = C(1) - hm;
#pragma unroll
    for (int q = 0; q < 9; q++) {
      const int d = 2 * q;
      const C wr = d < 6 ? wr1 : wr2;
      const C cu = cdot<C>(d, ux, uy, uz);
      C e = DEV ? wgt<C>(d) * (rho * (base + C(4.5) * (cu * cu)) - rho0) : wr * (base + C(4.5) * (cu * cu));
      C o = (C(3) * wr) * cu;
      // A = om_p (f+ - e), Bm = om_m (f- - o), f+- = (f_d +- f_d+1)/2
      C A = hp * (f[d] + f[d + 1]) - k.om_p * e;
      C Bm = hm * (f[d] - f[d + 1]) - k.om_m * o;
      if (FORCE) {
        const C w = wgt<C>(d);
        if (FORCE == 2 && cx(d) == 0) {  // c.F = 0
          A -= fac_p * w * m3uF;
        } else {
          const C cF = FORCE == 2 ? (cx(d) > 0 ? Fx : -Fx) : cdot<C>(d, Fx, Fy, Fz);
          A -= fac_p * w * (C(9) * (cu * cF) + m3uF);
          Bm -= fac_m * (C(3) * w) * cF;
        }
      }
      p[d] = (f[d] - A) - Bm;
      p[d + 1] = (f[d + 1] - A) + Bm;
    }
    C v = f[18] - k.om_p * (f[18] - (DEV ? wgt<C>(18) * (rho * base - rho0) : wr0 * base));
    if (FORCE) v += fac_p * wgt<C>(18) * m3uF;
    p[18] = v;
  }
}

// Wall velocity of the moving body at lattice point (px,py,pz).
__device__ __forceinline__ void wall_velocity(const Kinematics& k, double px, double py, double pz,
                                              double& wx, double& wy, double& wz) {
  const double rx = px - k.center[0], ry = py - k.center[1], rz = pz - k.center[2];
  wx = k.vel[0] + (k.omega[1] * rz - k.omega[2] * ry);
  wy = k.vel[1] + (k.omega[2] * rx - k.omega[0] * rz);
  wz = k.vel[2] + (k.omega[0] * ry - k.omega[1] * rx);
}

// Post-collision state of a node refilled with feq(rho0, u_wall(node)).  Not
// inlined: a fresh node and each of its old-fluid neighbours call the same code
// and therefore obtain bit-identical values.
template <class C, bool TRT, int FORCE>
__device__ __noinline__ void fresh_state(Coll<C> k, Kinematics kin, C rho0, int x, int y, int z,
                                         C* p, C* mom) {
  double wx, wy, wz;
  wall_velocity(kin, x + 0.5, y + 0.5, z + 0.5, wx, wy, wz);
  C f[Q];
#pragma unroll
  for (int d = 0; d < Q; d++) f[d] = feq<C>(d, rho0, C(wx), C(wy), C(wz));
  C rho, ux, uy, uz;
  moments<C, FORCE>(f, k, rho, ux, uy, uz);
  collide<C, TRT, FORCE>(f, p, k, rho, ux, uy, uz);
  mom[0] = rho;
  mom[1] = ux;
  mom[2] = uy;
  mom[3] = uz;
}

// ---- non-periodic faces -------------------------------------------------------------
// Incoming directions d (bit d) with c_d along `axis` equal to `sign`.
__host__ __device__ constexpr uint32_t dir_mask(int axis, int sign) {
  uint32_t m = 0;
  for (int d = 0; d < 18; d++) {
    const int c = axis == 0 ? cx(d) : (axis == 1 ? cy(d) : cz(d));
    if (c == sign) m |= 1u << d;
  }
  return m;
}

// Face situation of one node: bit d of `mask` is set when the source x - c_d of the
// incoming population d lies outside a non-periodic face.
struct FaceLane {
  uint32_t mask;
  bool xlo, xhi, ylo, yhi, zlo, zhi;
};

__device__ __forceinline__ FaceLane face_lane(const Grid& g, int x, int y, int z) {
  FaceLane f;
  f.xlo = !g.per[0] && x == 0;
  f.xhi = !g.per[0] && x == g.nx - 1;
  f.ylo = !g.per[1] && y == 0;
  f.yhi = !g.per[1] && y == g.ny - 1;
  f.zlo = !g.per[2] && z == 0;
  f.zhi = !g.per[2] && z == g.nz - 1;
  f.mask = (f.xlo ? dir_mask(0, 1) : 0u) | (f.xhi ? dir_mask(0, -1) : 0u) | (f.ylo ? dir_mask(1, 1) : 0u) |
           (f.yhi ? dir_mask(1, -1) : 0u) | (f.zlo ? dir_mask(2, 1) : 0u) | (f.zhi ? dir_mask(2, -1) : 0u);
  return f;
}

// Boundary value of incoming direction d whose source lies outside a non-periodic
// face (kept in the node's own slot A[d][x]).  At edges and corners the face of the
// x axis wins, then y, then z.  xlo/xhi/ylo/yhi: the node lies on that face.
// off: w_d rho0 when pst and the result are deviations (FP16 fast path), else 0.
template <class C>
__device__ __forceinline__ C face_value(const AAParams& p, const int d, const bool xlo, const bool xhi,
                                        const bool ylo, const bool yhi, const C rho, const C ux, const C uy,
                                        const C uz, const C* pst, const C off = C(0)) {
  const int o = opp(d);
  const bool xo = (cx(d) > 0 && xlo) || (cx(d) < 0 && xhi);
  const bool yo = (cy(d) > 0 && ylo) || (cy(d) < 0 && yhi);
  const int fx = cx(d) > 0 ? 0 : 1, fy = cy(d) > 0 ? 2 : 3, fz = cz(d) > 0 ? 4 : 5;
  // static indices only (the parameter block stays in the constant bank)
  const int kind = xo ? p.face_kind[fx] : (yo ? p.face_kind[fy] : p.face_kind[fz]);
  const C ufx = C(xo ? p.face_u[fx][0] : (yo ? p.face_u[fy][0] : p.face_u[fz][0]));
  const C ufy = C(xo ? p.face_u[fx][1] : (yo ? p.face_u[fy][1] : p.face_u[fz][1]));
  const C ufz = C(xo ? p.face_u[fx][2] : (yo ? p.face_u[fy][2] : p.face_u[fz][2]));
  if (kind == LBM_FACE_EQ_INLET) return feq<C>(d, rho, ufx, ufy, ufz) - off;
  if (kind == LBM_FACE_OUTFLOW) return pst[d];
  if (kind == LBM_FACE_PRESSURE) {
    const C cu = cdot<C>(d, ux, uy, uz);
    const C usq = ux * ux + uy * uy + uz * uz;
    return -pst[o] + C(2) * wgt<C>(d) * C(p.rho0) * (C(1) + C(4.5) * cu * cu - C(1.5) * usq) - C(2) * off;
  }
  return pst[o] - C(6) * wgt<C>(o) * rho * cdot<C>(o, ufx, ufy, ufz);
}

// ---- the step kernel ------------------------------------------------------------------
// General path of one fluid node: faces, solid links, moving-body refill, momentum
// exchange.  Kept out of line so that its register demand does not limit the
// occupancy of the interior fast path; only warps containing a boundary node run it.
template <class SP, bool ODD, bool TRT, int FORCE>
__device__ __noinline__ void aa_general(const AAParams& p, typename SP::S* __restrict__ A,
                                        const uint8_t* __restrict__ flags, const int x, const int y,
                                        const int z, const long long i, const uint8_t fl, double* acc,
                                        bool* has_out) {
  using C = typename SP::C;
  const Grid& g = p.g;
  const C rho0 = C(p.rho0);
  const Coll<C> k{C(p.omega_p), C(p.omega_m), C(p.gacc[0]), C(p.gacc[1]), C(p.gacc[2])};
  bool has_link = false;
  const long long nxl = g.nx, nxy = (long long)g.nx * g.ny;
  // neighbour coordinates; -1 when outside a non-periodic axis
  const int xs0 = x == 0 ? (g.per[0] ? g.nx - 1 : -1) : x - 1;
  const int xs2 = x == g.nx - 1 ? (g.per[0] ? 0 : -1) : x + 1;
  const int ys0 = y == 0 ? (g.per[1] ? g.ny - 1 : -1) : y - 1;
  const int ys2 = y == g.ny - 1 ? (g.per[1] ? 0 : -1) : y + 1;
  const int zs0 = z == 0 ? (g.per[2] ? g.nz - 1 : -1) : z - 1;
  const int zs2 = z == g.nz - 1 ? (g.per[2] ? 0 : -1) : z + 1;
  const int xs[3] = {xs0, x, xs2}, ys[3] = {ys0, y, ys2}, zs[3] = {zs0, z, zs2};
  const bool on_face = (xs0 | xs2 | ys0 | ys2 | zs0 | zs2) < 0;
  const bool near = (fl & F_NEAR) != 0;

  uint32_t face = 0, bcp = 0, bcc = 0, mov = 0;
  if (on_face || near) {
#pragma unroll
    for (int d = 0; d < 18; d++) {
      const int sx = xs[1 - cx(d)], sy = ys[1 - cy(d)], sz = zs[1 - cz(d)];
      if ((sx | sy | sz) < 0) {
        face |= 1u << d;
      } else if (near) {
        const uint8_t fs = flags[sx + nxl * sy + nxy * sz];
        if (fs & F_SOLID_PREV) bcp |= 1u << d;
        if (fs & F_SOLID) bcc |= 1u << d;
        if (fs & F_MOVING) mov |= 1u << d;
      }
    }
  }
  const uint32_t bcr = face | bcp;  // incoming slots holding boundary values (read side)
  const uint32_t bcw = face | bcc;  // incoming slots to fill with boundary values (write side)
  const bool fresh = (fl & F_SOLID_PREV) != 0;

  C pst[Q];
  C rho, ux, uy, uz;
  if (!fresh) {
    C f[Q];
#pragma unroll
    for (int d = 0; d < Q; d++) {
      long long a;
      if (!ODD || d == 18) {
        a = (long long)d * g.plane + i;
      } else {
        const long long src = xs[1 - cx(d)] + nxl * ys[1 - cy(d)] + nxy * zs[1 - cz(d)];
        a = ((bcr >> d) & 1u) ? (long long)d * g.plane + i : (long long)opp(d) * g.plane + src;
      }
      f[d] = SP::ld(A + a, d, rho0);
    }
    moments<C, FORCE>(f, k, rho, ux, uy, uz);
    collide<C, TRT, FORCE>(f, pst, k, rho, ux, uy, uz);
  } else {
    C mom[4];
    fresh_state<C, TRT, FORCE>(k, p.kin, rho0, x, y, z, pst, mom);
    rho = mom[0];
    ux = mom[1];
    uy = mom[2];
    uz = mom[3];
  }

  // boundary value of incoming direction d (own slot A[d][x])
  auto bcval = [&](const int d) -> C {
    const int o = opp(d);
    if ((face >> d) & 1u) return face_value<C>(p, d, xs0 < 0, xs2 < 0, ys0 < 0, ys2 < 0, rho, ux, uy, uz, pst);
    C cdu = C(0);
    if ((mov >> d) & 1u) {
      double wx, wy, wz;
      wall_velocity(p.kin, x + 0.5 + 0.5 * cx(o), y + 0.5 + 0.5 * cy(o), z + 0.5 + 0.5 * cz(o), wx,
                    wy, wz);
      cdu = cdot<C>(o, C(wx), C(wy), C(wz));
    }
    const C v = pst[o] - C(6) * wgt<C>(o) * rho * cdu;
    if (p.compute_force) {
      // momentum exchange of link (x, o): c_o (f*_o + f_in)
      const double t = (double)pst[o] + (double)v;
      const double fx = t * cx(o), fy = t * cy(o), fz = t * cz(o);
      const double rx = x + 0.5 + 0.5 * cx(o) - p.kin.center[0];
      const double ry = y + 0.5 + 0.5 * cy(o) - p.kin.center[1];
      const double rz = z + 0.5 + 0.5 * cz(o) - p.kin.center[2];
      acc[0] += fx;
      acc[1] += fy;
      acc[2] += fz;
      acc[3] += ry * fz - rz * fy;
      acc[4] += rz * fx - rx * fz;
      acc[5] += rx * fy - ry * fx;
      has_link = true;
    }
    return v;
  };

  if (!ODD) {
#pragma unroll
    for (int d = 0; d < Q; d++) {
      C v;
      if ((bcw >> d) & 1u) v = bcval(d);
      else v = pst[opp(d)];
      SP::st(A + (long long)d * g.plane + i, v, d, rho0);
    }
  } else {
#pragma unroll
    for (int j = 0; j < Q; j++) {
      const int o = opp(j);
      if ((bcw >> o) & 1u) {
        // target x + c_j is outside/solid: the boundary value of incoming o goes to A[o][x]
        const C v = bcval(o);
        SP::st(A + (long long)o * g.plane + i, v, o, rho0);
      } else if (j == 18 || !fresh || ((bcp >> o) & 1u)) {
        // a fresh node leaves its emission toward old-fluid targets to them
        const long long tgt = xs[1 + cx(j)] + nxl * ys[1 + cy(j)] + nxy * zs[1 + cz(j)];
        SP::st(A + (long long)j * g.plane + tgt, pst[j], j, rho0);
      }
    }
    if (!fresh) {
      const uint32_t fnb = bcp & ~bcc & ~face;  // neighbours uncovered this step
      if (fnb) {
#pragma unroll
        for (int d = 0; d < 18; d++) {
          if (!((fnb >> d) & 1u)) continue;
          // source coordinates of direction d (x - c_d), wrapped
          const int sx = xs[1 - cx(d)], sy = ys[1 - cy(d)], sz = zs[1 - cz(d)];
          C q[Q], mom[4];
          fresh_state<C, TRT, FORCE>(k, p.kin, rho0, sx, sy, sz, q, mom);
          C qd = q[0];
#pragma unroll
          for (int e = 1; e < Q; e++)
            if (e == d) qd = q[e];
          SP::st(A + (long long)d * g.plane + i, qd, d, rho0);
        }
      }
    }
  }
  *has_out = *has_out || has_link;
}

// Fast path: a node whose only boundaries are static no-slip links (bc = incoming
// directions whose source is solid; 0 for most nodes) and, with FACES, non-periodic
// faces (face = incoming directions whose source lies outside the box).  Neighbour
// offsets are precomputed on the host (p.off_rd / p.off_wr); the periodic x wrap is
// patched per lane.  A static no-slip bounce-back value for incoming d is
// f*_{opp(d)}: in the even phase that is exactly the swapped store, in the odd phase
// it only redirects the store of f*_j from the solid target x + c_j to the own slot
// opp(j).  Face values follow face_value(), also through the own slots.
//
// The loads are split from the compute so that the caller can issue them before the
// node's flag byte arrives (speculatively, for every lane whose coordinates allow
// the fast path), instead of chaining two memory round trips.
// Fast-path population access: the stored value itself when the storage keeps
// deviations (computed in deviation form), the population otherwise.
template <class SP>
__device__ __forceinline__ typename SP::C ld_fast(const typename SP::S* p, int d, typename SP::C rho0) {
  if (SP::DEV) return SP::ld_raw(p);
  return SP::ld(p, d, rho0);
}
template <class SP>
__device__ __forceinline__ void st_fast(typename SP::S* p, typename SP::C v, int d, typename SP::C rho0) {
  if (SP::DEV)
    SP::st_raw(p, v);
  else
    SP::st(p, v, d, rho0);
}

template <bool FACES>
__device__ __forceinline__ void x_wrap_fix(const Grid& g, const int x, long long& fix_lo, long long& fix_hi) {
  const bool per = FACES ? g.per[0] != 0 : true;  // without FACES every axis is periodic
  fix_lo = (per && x == 0) ? (long long)g.nx : 0;
  fix_hi = (per && x == g.nx - 1) ? (long long)g.nx : 0;
}

template <class SP, bool ODD, bool FACES>
__device__ __forceinline__ void aa_fast_load(const AAParams& p, const typename SP::S* __restrict__ base,
                                             const int x, const uint32_t face, typename SP::C* f) {
  using C = typename SP::C;
  const C rho0 = C(p.rho0);
  long long fix_lo = 0, fix_hi = 0;  // periodic x wrap at the row ends (odd phase)
  if (ODD) x_wrap_fix<FACES>(p.g, x, fix_lo, fix_hi);
#pragma unroll
  for (int d = 0; d < Q; d++) {
    long long o = p.off_rd[d];
    if (ODD) {
      if (cx(d) == 1) o += fix_lo;
      if (cx(d) == -1) o -= fix_hi;
      // source outside a face: the boundary value sits in the own slot
      if (FACES && d < 18 && ((face >> d) & 1u)) o = (long long)d * p.g.plane;
    }
    f[d] = ld_fast<SP>(base + o, d, rho0);
  }
}

// Momentum exchange of one cell's static bounce-back links (bit d of bc: incoming d, source
// solid): each link o = opp(d) carries c_o (f*_o + f*_o).  The links' torque is r_cell x
// F_cell with r_cell the cell centre relative to the torque centre: the half-link offsets
// 0.5 c_o drop out because c_o x c_o = 0, so a link costs one addition per nonzero component.
// FP16-deviation storage keeps a cross product per link: with the per-cell form the inlined
// code made the eight-cell even kernel 12 % slower on B200 even with the force off.
template <class SP>
__device__ __forceinline__ void pair_links(const AAParams& p, const int x, const int y, const int z, const uint32_t bc,
                                           const typename SP::C* pst, double* acc) {
  using C = typename SP::C;
  if constexpr (SP::DEV) {
#pragma unroll
    for (int d = 0; d < 18; d++) {
      if (!((bc >> d) & 1u)) continue;
      const int o = opp(d);
      const double t = 2.0 * (double)(pst[o] + wgt<C>(o) * C(p.rho0));
      const double fx = t * cx(o), fy = t * cy(o), fz = t * cz(o);
      const double rx = x + 0.5 + 0.5 * cx(o) - p.kin.center[0];
      const double ry = y + 0.5 + 0.5 * cy(o) - p.kin.center[1];
      const double rz = z + 0.5 + 0.5 * cz(o) - p.kin.center[2];
      acc[0] += fx;
      acc[1] += fy;
      acc[2] += fz;
      acc[3] += ry * fz - rz * fy;
      acc[4] += rz * fx - rx * fz;
      acc[5] += rx * fy - ry * fx;
    }
    return;
  }
  double fx = 0.0, fy = 0.0, fz = 0.0;
#pragma unroll
  for (int d = 0; d < 18; d++) {
    if (!((bc >> d) & 1u)) continue;
    const int o = opp(d);
    const double t = 2.0 * (double)pst[o];
    if (cx(o) > 0) fx += t;
    if (cx(o) < 0) fx -= t;
    if (cy(o) > 0) fy += t;
    if (cy(o) < 0) fy -= t;
    if (cz(o) > 0) fz += t;
    if (cz(o) < 0) fz -= t;
  }
  const double rx = x + 0.5 - p.kin.center[0];
  const double ry = y + 0.5 - p.kin.center[1];
  const double rz = z + 0.5 - p.kin.center[2];
  acc[0] += fx;
  acc[1] += fy;
  acc[2] += fz;
  acc[3] += ry * fz - rz * fy;
  acc[4] += rz * fx - rx * fz;
  acc[5] += rx * fy - ry * fx;
}

template <class SP, bool ODD, bool TRT, int FORCE, bool FACES>
__device__ __forceinline__ void aa_fast_finish(const AAParams& p, typename SP::S* __restrict__ base,
                                               const int x, const int y, const int z, const uint32_t bc,
                                               const FaceLane& fc, typename SP::C* f, double* acc,
                                               bool* has_link) {
  using C = typename SP::C;
  const C rho0 = C(p.rho0);
  const Coll<C> k{C(p.omega_p), C(p.omega_m), C(p.gacc[0]), C(p.gacc[1]), C(p.gacc[2])};
  if (ODD && bc) {  // bounce-back values are kept in the own slots
#pragma unroll
    for (int d = 0; d < 18; d++)
      if ((bc >> d) & 1u) f[d] = ld_fast<SP>(base + (long long)d * p.g.plane, d, rho0);
  }
  long long fix_lo = 0, fix_hi = 0;
  if (ODD) x_wrap_fix<FACES>(p.g, x, fix_lo, fix_hi);
  C rho, ux, uy, uz;
  moments<C, FORCE, SP::DEV>(f, k, rho, ux, uy, uz, rho0);
  C pst[Q];
  collide<C, TRT, FORCE, SP::DEV>(f, pst, k, rho, ux, uy, uz, rho0);
  const uint32_t face = FACES ? fc.mask : 0u;
  // warps without a face node take the plain store loop; a warp with one runs the
  // per-direction face test on every lane (one loop, no divergence between loops)
  if (FACES && __any_sync(__activemask(), face != 0u)) {
    // Every direction is stored without a branch; an incoming direction whose source lies
    // outside (j in the even phase, opp(j) in the odd phase) goes to the node's own slot
    // with a placeholder.  The face values follow, one divergent branch per face rather
    // than one per direction, faces in ascending priority so that at edges and corners
    // the value of face_value's rule (x face, then y, then z) is stored last.
#pragma unroll
    for (int j = 0; j < Q; j++) {
      long long o = p.off_wr[j];
      if (ODD) {
        if (cx(j) == 1) o -= fix_hi;
        if (cx(j) == -1) o += fix_lo;
        if (j < 18 && (((face | bc) >> opp(j)) & 1u)) o = (long long)opp(j) * p.g.plane;
      }
      st_fast<SP>(base + o, ODD ? pst[j] : pst[opp(j)], j, rho0);
    }
    const auto fix = [&](const int axis, const int sign, const bool xl, const bool xh, const bool yl, const bool yh) {
#pragma unroll
      for (int d = 0; d < 18; d++) {
        if ((axis == 0 ? cx(d) : (axis == 1 ? cy(d) : cz(d))) != sign) continue;
        const C v = face_value<C>(p, d, xl, xh, yl, yh, rho, ux, uy, uz, pst, SP::DEV ? wgt<C>(d) * rho0 : C(0));
        st_fast<SP>(base + (long long)d * p.g.plane, v, d, rho0);
      }
    };
    if (fc.zlo) fix(2, 1, false, false, false, false);
    if (fc.zhi) fix(2, -1, false, false, false, false);
    if (fc.ylo) fix(1, 1, false, false, true, false);
    if (fc.yhi) fix(1, -1, false, false, false, true);
    if (fc.xlo) fix(0, 1, true, false, false, false);
    if (fc.xhi) fix(0, -1, false, true, false, false);
  } else {
#pragma unroll
    for (int j = 0; j < Q; j++) {
      long long o = p.off_wr[j];
      if (ODD) {
        if (cx(j) == 1) o -= fix_hi;
        if (cx(j) == -1) o += fix_lo;
        if (j < 18 && ((bc >> opp(j)) & 1u)) o = (long long)opp(j) * p.g.plane;
      }
      st_fast<SP>(base + o, ODD ? pst[j] : pst[opp(j)], j, rho0);
    }
  }
  if (bc && p.compute_force) {
    pair_links<SP>(p, x, y, z, bc, pst, acc);  // momentum exchange of the static links
    *has_link = true;
  }
}

// Ghost plane on a halo face (z-slab decomposition).  The step kernels put one z plane in
// a block, so a ghost block leaves at once; the batched kernel checks per node.
__device__ __forceinline__ bool ghost_plane(const AAParams& p, const int z) {
  return (z == 0 && p.face_kind[4] == LBM_FACE_HALO) || (z == p.g.nz - 1 && p.face_kind[5] == LBM_FACE_HALO);
}

// One node on the direct path: lanes whose coordinates allow the fast path issue
// their population loads at once; the flag byte (and, next to a solid, the link
// word) decides afterwards whether the warp finishes on the fast path or reruns the
// node on the general path.  All 32 lanes of a warp reach the vote.
//
// Coordinates that allow the fast path: even phase — every node (own slots only);
// odd phase — every node except the rows next to a periodic y or z wrap (their
// neighbour offsets wrap).  Without FACES (all axes periodic) the same rule holds;
// with FACES, nodes on non-periodic faces are fast too (face mask).
template <class SP, bool ODD, bool TRT, int FORCE, bool FACES>
__device__ __forceinline__ void aa_direct(const AAParams& p, typename SP::S* __restrict__ A,
                                          const uint8_t* __restrict__ flags, const int x, const int y, const int z,
                                          const bool inb, double* acc, bool* has_link) {
  using C = typename SP::C;
  const Grid& g = p.g;
  const long long i = inb ? node_index(g, x, y, z) : 0;
  FaceLane fc{0u, false, false, false, false, false, false};
  bool coord_fast;
  if (FACES) {
    if (inb) fc = face_lane(g, x, y, z);
    coord_fast = inb;
    if (ODD) coord_fast = coord_fast && (!g.per[1] || (y > 0 && y < g.ny - 1)) && (!g.per[2] || (z > 0 && z < g.nz - 1));
  } else {
    const bool xin = g.per[0] || (x > 0 && x < g.nx - 1);
    coord_fast = inb && xin;
    if (ODD) {
      coord_fast = coord_fast && y > 0 && y < g.ny - 1 && z > 0 && z < g.nz - 1;
    } else {
      coord_fast = coord_fast && (g.per[1] || (y > 0 && y < g.ny - 1)) && (g.per[2] || (z > 0 && z < g.nz - 1));
    }
  }
  const uint8_t fl = inb ? flags[i] : (uint8_t)F_SOLID;
  C f[Q];
  if (coord_fast) aa_fast_load<SP, ODD, FACES>(p, A + i, x, fc.mask, f);
  // the ghost plane on a halo face (z-slab decomposition) is read and written by its
  // neighbours like any fluid or solid node but never updated itself
  const bool ghost = FACES && inb &&
                     ((z == 0 && p.face_kind[4] == LBM_FACE_HALO) || (z == g.nz - 1 && p.face_kind[5] == LBM_FACE_HALO));
  const bool solid = (fl & F_SOLID) != 0 || ghost;
  // fast when the only boundaries are static no-slip links (link word: current ==
  // previous links, no moving-body link, not uncovered)
  uint32_t bc = 0;
  bool static_links = true;
  if (!solid && (fl & F_NEAR)) {
    const unsigned long long lw = p.links[i];
    const uint32_t cur = (uint32_t)(lw & 0x3FFFFu), prev = (uint32_t)((lw >> 18) & 0x3FFFFu);
    const uint32_t mov = (uint32_t)((lw >> 36) & 0x3FFFFu);
    static_links = cur == prev && mov == 0 && !(fl & F_SOLID_PREV);
    bc = cur;
  }
  const bool fast = coord_fast && static_links;
  const bool warp_fast = __all_sync(0xffffffffu, solid || fast);
  if (warp_fast) {
    if (!solid) aa_fast_finish<SP, ODD, TRT, FORCE, FACES>(p, A + i, x, y, z, bc, fc, f, acc, has_link);
  } else if (!solid) {
    aa_general<SP, ODD, TRT, FORCE>(p, A, flags, x, y, z, i, fl, acc, has_link);
  }
}

template <class SP, bool ODD, bool TRT, int FORCE, bool FACES>
__global__ void __launch_bounds__(256, SP::MIN_BLOCKS) aa_step_kernel(const __grid_constant__ AAParams p,
                                                                      typename SP::S* __restrict__ A,
                                                                      const uint8_t* __restrict__ flags) {
  const Grid& g = p.g;
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  const int y = blockIdx.y * blockDim.y + threadIdx.y;
  const int z = blockIdx.z;
  const bool inb = (x < g.nx) && (y < g.ny);
  clear_record(p.zero_next);  // the next step's force record (read by the next launch only)
  if (ghost_plane(p, z)) return;  // whole block in a ghost plane
  double acc[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
  bool has_link = false;
  aa_direct<SP, ODD, TRT, FORCE, FACES>(p, A, flags, x, y, z, inb, acc, &has_link);
  if (p.compute_force) block_force_reduce(acc, has_link, p.force + block_stripe());
}

// ---- pair kernel (fully periodic boxes, nx a multiple of 128) ---------------------------
// One thread updates the two x-adjacent cells (x0, x0+1), x0 even.  The two cells' slots
// of a direction are adjacent and aligned to twice the element size whenever the
// direction has no x component (all 19 in the even phase, 9 in the odd phase): those
// move as one two-element word (half2 / float2 / double2); the x-shifted ones move as
// two elements.  Addressing and control are shared by the pair and every thread keeps
// more loads in flight.  Warps that meet a non-static boundary rerun both cells on the
// general path; a solid cell's own slots are never read by anyone, so an even-phase
// two-element store may overwrite them.
template <class S>
struct Pair2;
template <>
struct Pair2<__half> {
  static __device__ __forceinline__ void ld(const __half* p, float& a, float& b) {
    const __half2 h = *reinterpret_cast<const __half2*>(p);
    a = __low2float(h);
    b = __high2float(h);
  }
  static __device__ __forceinline__ void st(__half* p, float a, float b) {
    *reinterpret_cast<__half2*>(p) = __floats2half2_rn(a, b);
  }
};
template <>
struct Pair2<float> {
  static __device__ __forceinline__ void ld(const float* p, float& a, float& b) {
    const float2 v = *reinterpret_cast<const float2*>(p);
    a = v.x;
    b = v.y;
  }
  static __device__ __forceinline__ void st(float* p, float a, float b) { *reinterpret_cast<float2*>(p) = make_float2(a, b); }
};
template <>
struct Pair2<double> {
  static __device__ __forceinline__ void ld(const double* p, double& a, double& b) {
    const double2 v = *reinterpret_cast<const double2*>(p);
    a = v.x;
    b = v.y;
  }
  static __device__ __forceinline__ void st(double* p, double a, double b) {
    *reinterpret_cast<double2*>(p) = make_double2(a, b);
  }
};

template <class SP, bool ODD, bool TRT, int FORCE>
__device__ __forceinline__ void pair_cell(const AAParams& p, const typename SP::C* f, typename SP::C* pst) {
  using C = typename SP::C;
  const Coll<C> k{C(p.omega_p), C(p.omega_m), C(p.gacc[0]), C(p.gacc[1]), C(p.gacc[2])};
  const C rho0 = C(p.rho0);
  C rho, ux, uy, uz;
  moments<C, FORCE, SP::DEV>(f, k, rho, ux, uy, uz, rho0);
  collide<C, TRT, FORCE, SP::DEV>(f, pst, k, rho, ux, uy, uz, rho0);
}

// The update of the cell pair (x0, x0 + 1), x0 even, as described above; all 32 lanes of the
// warp take part (warp vote).
template <class SP, bool ODD, bool TRT, int FORCE>
__device__ __forceinline__ void pair_cells(const AAParams& p, typename SP::S* __restrict__ A,
                                           const uint8_t* __restrict__ flags, const int x0, const int y, const int z,
                                           const bool inb, double* acc, bool& has_link) {
  using S = typename SP::S;
  using C = typename SP::C;
  const Grid& g = p.g;
  const long long i0 = inb ? node_index(g, x0, y, z) : 0;
  const bool coord_fast = inb && (!ODD || (y > 0 && y < g.ny - 1 && z > 0 && z < g.nz - 1));
  uint32_t fl0 = F_SOLID, fl1 = F_SOLID;
  if (inb) {
    const uint32_t fw = *reinterpret_cast<const unsigned short*>(flags + i0);
    fl0 = fw & 0xFFu;
    fl1 = fw >> 8;
  }
  const long long fix_lo = x0 == 0 ? (long long)g.nx : 0;            // cell 0 at x = 0
  const long long fix_hi = x0 + 1 == g.nx - 1 ? (long long)g.nx : 0;  // cell 1 at x = nx - 1
  C f0[Q], f1[Q];
  // byte bases: the cell pair, and each cell with its periodic x wrap folded in; with the
  // byte offsets of the parameter block each access is one 64-bit add (FP32 on B200:
  // odd phase -2.6 %, even -0.6 % against element offsets)
  const char* const Bi = reinterpret_cast<const char*>(A + i0);
  const char* const B0 = reinterpret_cast<const char*>(A + i0 + fix_lo);
  const char* const B1 = reinterpret_cast<const char*>(A + i0 + 1 - fix_hi);
  if (coord_fast) {
#pragma unroll
    for (int d = 0; d < Q; d++) {
      const long long o = p.offb_rd[d];
      if (!ODD || cx(d) == 0) {
        Pair2<S>::ld(reinterpret_cast<const S*>(Bi + o), f0[d], f1[d]);
      } else if (cx(d) == 1) {
        f0[d] = ld_fast<SP>(reinterpret_cast<const S*>(B0 + o), d, C(p.rho0));
        f1[d] = ld_fast<SP>(reinterpret_cast<const S*>(Bi + o) + 1, d, C(p.rho0));
      } else {
        f0[d] = ld_fast<SP>(reinterpret_cast<const S*>(Bi + o), d, C(p.rho0));
        f1[d] = ld_fast<SP>(reinterpret_cast<const S*>(B1 + o), d, C(p.rho0));
      }
    }
  }
  const bool solid0 = (fl0 & F_SOLID) != 0, solid1 = (fl1 & F_SOLID) != 0;
  uint32_t bc0 = 0, bc1 = 0;
  bool st0 = true, st1 = true;
  if (!solid0 && (fl0 & F_NEAR)) {
    const unsigned long long lw = p.links[i0];
    bc0 = (uint32_t)(lw & 0x3FFFFu);
    st0 = bc0 == (uint32_t)((lw >> 18) & 0x3FFFFu) && ((lw >> 36) & 0x3FFFFu) == 0 && !(fl0 & F_SOLID_PREV);
  }
  if (!solid1 && (fl1 & F_NEAR)) {
    const unsigned long long lw = p.links[i0 + 1];
    bc1 = (uint32_t)(lw & 0x3FFFFu);
    st1 = bc1 == (uint32_t)((lw >> 18) & 0x3FFFFu) && ((lw >> 36) & 0x3FFFFu) == 0 && !(fl1 & F_SOLID_PREV);
  }
  const bool both_solid = solid0 && solid1;
  const bool fast = coord_fast && st0 && st1;
  if (__all_sync(0xffffffffu, both_solid || fast)) {
    if (!both_solid) {
      if (ODD && (bc0 | bc1)) {  // bounce-back values are kept in the own slots
#pragma unroll
        for (int d = 0; d < 18; d++) {
          if ((bc0 >> d) & 1u) f0[d] = ld_fast<SP>(A + (long long)d * g.plane + i0, d, C(p.rho0));
          if ((bc1 >> d) & 1u) f1[d] = ld_fast<SP>(A + (long long)d * g.plane + i0 + 1, d, C(p.rho0));
        }
      }
      C p0[Q], p1[Q];
      if (!solid0) {
        pair_cell<SP, ODD, TRT, FORCE>(p, f0, p0);
      } else {
#pragma unroll
        for (int d = 0; d < Q; d++) p0[d] = C(0);
      }
      if (!solid1) {
        pair_cell<SP, ODD, TRT, FORCE>(p, f1, p1);
      } else {
#pragma unroll
        for (int d = 0; d < Q; d++) p1[d] = C(0);
      }
      const bool plain = !solid0 && !solid1 && !(bc0 | bc1);
      const C rho0 = C(p.rho0);
      if (ODD && plain) {
        // both cells fluid without links: one loop without per-direction branches
        // (FP32 odd phase 4.23 -> 3.85 ms at 512^3 on B200)
#pragma unroll
        for (int j = 0; j < Q; j++) {
          const long long o = p.offb_wr[j];
          char* const bi = const_cast<char*>(Bi) + o;
          if (cx(j) == 0) {
            Pair2<S>::st(reinterpret_cast<S*>(bi), p0[j], p1[j]);
          } else if (cx(j) == 1) {
            st_fast<SP>(reinterpret_cast<S*>(bi), p0[j], j, rho0);
            st_fast<SP>(reinterpret_cast<S*>(const_cast<char*>(B1) + o), p1[j], j, rho0);
          } else {
            st_fast<SP>(reinterpret_cast<S*>(const_cast<char*>(B0) + o), p0[j], j, rho0);
            st_fast<SP>(reinterpret_cast<S*>(bi) + 1, p1[j], j, rho0);
          }
        }
      } else {
#pragma unroll
        for (int j = 0; j < Q; j++) {
          if (!ODD) {  // own slots of both cells: one word
            Pair2<S>::st(A + (long long)j * g.plane + i0, p0[opp(j)], p1[opp(j)]);
            continue;
          }
          const long long o = p.off_wr[j];
          const int oj = opp(j);
          if (cx(j) == 0 && plain) {
            Pair2<S>::st(A + i0 + o, p0[j], p1[j]);
            continue;
          }
          if (!solid0) {
            long long a = i0 + o + (cx(j) == -1 ? fix_lo : 0);
            if (j < 18 && ((bc0 >> oj) & 1u)) a = (long long)oj * g.plane + i0;
            st_fast<SP>(A + a, p0[j], j, rho0);
          }
          if (!solid1) {
            long long a = i0 + 1 + o - (cx(j) == 1 ? fix_hi : 0);
            if (j < 18 && ((bc1 >> oj) & 1u)) a = (long long)oj * g.plane + i0 + 1;
            st_fast<SP>(A + a, p1[j], j, rho0);
          }
        }
      }
      if (p.compute_force && (bc0 | bc1)) {
        pair_links<SP>(p, x0, y, z, bc0, p0, acc);
        pair_links<SP>(p, x0 + 1, y, z, bc1, p1, acc);
        has_link = true;
      }
    }
  } else {
    if (inb && !solid0) aa_general<SP, ODD, TRT, FORCE>(p, A, flags, x0, y, z, i0, (uint8_t)fl0, acc, &has_link);
    if (inb && !solid1) aa_general<SP, ODD, TRT, FORCE>(p, A, flags, x0 + 1, y, z, i0 + 1, (uint8_t)fl1, acc, &has_link);
  }
}

template <class SP, bool ODD, bool TRT, int FORCE>
__global__ void __launch_bounds__(256, (SP::MIN_BLOCKS > 2 ? 3 : 1)) aa_pair_kernel(const __grid_constant__ AAParams p,
                                                                                typename SP::S* __restrict__ A,
                                                                                const uint8_t* __restrict__ flags) {
  const Grid& g = p.g;
  const int x0 = 2 * (blockIdx.x * blockDim.x + threadIdx.x);
  const int y = blockIdx.y * blockDim.y + threadIdx.y;
  const int z = blockIdx.z;
  const bool inb = x0 < g.nx && y < g.ny;
  clear_record(p.zero_next);
  if (ghost_plane(p, z)) return;  // whole block in a ghost plane
  double acc[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
  bool has_link = false;
  pair_cells<SP, ODD, TRT, FORCE>(p, A, flags, x0, y, z, inb, acc, has_link);
  if (p.compute_force) block_force_reduce(acc, has_link, p.force + block_stripe());
}

// Odd phase of the pair kernel with every direction moved as one aligned two-element word
// per thread (FP32 storage): an x-shifted direction takes the word of the thread's own two
// positions, the element that enters from the neighbouring thread comes by warp shuffle,
// and only the warp's edge lanes (0 and 31) move one more element through memory, with the
// periodic x wrap.  Each slot is read and written by exactly one thread: an aligned word a
// warp covers only in part gets its missing element from the neighbouring warp's edge lane.
// Warps holding a solid, near-boundary or uncovered cell, or a row next to a y/z wrap, run
// the pair update above.
template <class SP, bool TRT, int FORCE>
__global__ void __launch_bounds__(256, (SP::MIN_BLOCKS > 2 ? 3 : 1)) aa_pair_odd_kernel(const __grid_constant__ AAParams p,
                                                                                    typename SP::S* __restrict__ A,
                                                                                    const uint8_t* __restrict__ flags) {
  using S = typename SP::S;
  using C = typename SP::C;
  static_assert(sizeof(S) == 4 && !SP::DEV, "FP32 storage");
  const Grid& g = p.g;
  const int lane = threadIdx.x & 31;  // blockDim.x is a multiple of 32: a warp is 64 cells of a row
  const int x0 = 2 * (blockIdx.x * blockDim.x + threadIdx.x);
  const int y = blockIdx.y * blockDim.y + threadIdx.y;
  const int z = blockIdx.z;
  const bool inb = x0 < g.nx && y < g.ny;
  clear_record(p.zero_next);
  if (ghost_plane(p, z)) return;  // whole block in a ghost plane
  double acc[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
  bool has_link = false;
  const long long i0 = inb ? node_index(g, x0, y, z) : 0;
  uint32_t fw = 0x0101u * F_SOLID;
  if (inb) fw = *reinterpret_cast<const unsigned short*>(flags + i0);
  // two fluid cells away from any solid (F_SOLID, F_SOLID_PREV, F_NEAR clear), not in a row
  // next to the y/z wrap
  const bool plain = inb && y > 0 && y < g.ny - 1 && z > 0 && z < g.nz - 1 && (fw & 0x0707u) == 0u;
  if (__all_sync(0xffffffffu, plain)) {
    constexpr long long E = sizeof(S);
    char* const Ai = reinterpret_cast<char*>(A + i0);
    const long long wrap_lo = x0 == 0 ? E * g.nx : 0;          // element x0 - 1 at x = nx - 1
    const long long wrap_hi = x0 + 2 == g.nx ? E * g.nx : 0;   // element x0 + 2 at x = 0
    C f0[Q], f1[Q];
    C edge[Q];
#pragma unroll
    for (int d = 0; d < Q; d++) {
      const long long o = p.offb_rd[d];
      if (cx(d) == 0) {
        const float2 v = *reinterpret_cast<const float2*>(Ai + o);
        f0[d] = v.x;
        f1[d] = v.y;
      } else if (cx(d) == 1) {  // pull from x - 1: o addresses element x0 - 1 of the source row
        const float2 v = *reinterpret_cast<const float2*>(Ai + o + E);
        f0[d] = v.y;  // replaced by the previous lane's second element below
        f1[d] = v.x;
        if (lane == 0) edge[d] = *reinterpret_cast<const S*>(Ai + o + wrap_lo);
      } else {  // pull from x + 1: o addresses element x0 + 1
        const float2 v = *reinterpret_cast<const float2*>(Ai + o - E);
        f0[d] = v.y;
        f1[d] = v.x;  // replaced by the next lane's first element below
        if (lane == 31) edge[d] = *reinterpret_cast<const S*>(Ai + o + E - wrap_hi);
      }
    }
#pragma unroll
    for (int d = 0; d < Q; d++) {
      if (cx(d) == 1) {
        const C up = __shfl_up_sync(0xffffffffu, f0[d], 1);
        f0[d] = lane == 0 ? edge[d] : up;
      } else if (cx(d) == -1) {
        const C dn = __shfl_down_sync(0xffffffffu, f1[d], 1);
        f1[d] = lane == 31 ? edge[d] : dn;
      }
    }
    C p0[Q], p1[Q];
    pair_cell<SP, true, TRT, FORCE>(p, f0, p0);
    pair_cell<SP, true, TRT, FORCE>(p, f1, p1);
#pragma unroll
    for (int j = 0; j < Q; j++) {
      const long long o = p.offb_wr[j];
      if (cx(j) == 0) {
        *reinterpret_cast<float2*>(Ai + o) = make_float2(p0[j], p1[j]);
      } else if (cx(j) == 1) {  // push to x + 1: o addresses element x0 + 1 of the target row
        const C up = __shfl_up_sync(0xffffffffu, p1[j], 1);
        if (lane != 0)
          *reinterpret_cast<float2*>(Ai + o - E) = make_float2(up, p0[j]);
        else  // element x0 comes from the previous warp's lane 31
          *reinterpret_cast<S*>(Ai + o) = p0[j];
        if (lane == 31) *reinterpret_cast<S*>(Ai + o + E - wrap_hi) = p1[j];
      } else {  // push to x - 1: o addresses element x0 - 1
        const C dn = __shfl_down_sync(0xffffffffu, p0[j], 1);
        if (lane != 31)
          *reinterpret_cast<float2*>(Ai + o + E) = make_float2(p1[j], dn);
        else  // element x0 + 1 comes from the next warp's lane 0
          *reinterpret_cast<S*>(Ai + o + E) = p1[j];
        if (lane == 0) *reinterpret_cast<S*>(Ai + o + wrap_lo) = p0[j];
      }
    }
  } else {
    pair_cells<SP, true, TRT, FORCE>(p, A, flags, x0, y, z, inb, acc, has_link);
  }
  if (p.compute_force) block_force_reduce(acc, has_link, p.force + block_stripe());
}

// Odd-phase variant of the pair kernel (FP16-deviation storage): a cell's odd-phase
// writes are read back only by the same cell in the next step, so cell 0 stores its
// x-shifted outputs before cell 1 collides and only the nine values that pair with
// cell 1 stay live.  Row bases with the periodic x wrap folded in keep the addressing
// to one add per access.  Measured on B200 (512^3 porous box): 11 % faster than the
// joint pair kernel for FP16 storage; slower for FP32 and for the even phase, which
// keep aa_pair_kernel.
// The odd-phase update of the cell pair (x0, x0 + 1), x0 even, as described above; all 32
// lanes of the warp take part (warp vote).
template <class SP, bool TRT, int FORCE>
__device__ __forceinline__ void pair_split_cells(const AAParams& p, typename SP::S* __restrict__ A,
                                                 const uint8_t* __restrict__ flags, const int x0, const int y,
                                                 const int z, const bool inb, double* acc, bool& has_link) {
  using S = typename SP::S;
  using C = typename SP::C;
  const Grid& g = p.g;
  const long long i0 = inb ? node_index(g, x0, y, z) : 0;
  const bool coord_fast = inb && y > 0 && y < g.ny - 1 && z > 0 && z < g.nz - 1;
  uint32_t fl0 = F_SOLID, fl1 = F_SOLID;
  if (inb) {
    const uint32_t fw = *reinterpret_cast<const unsigned short*>(flags + i0);
    fl0 = fw & 0xFFu;
    fl1 = fw >> 8;
  }
  // Row bases with the periodic x wrap folded in: cell 0 at x = 0 reaches x = -1 at
  // x = nx - 1 (pull with c_x = +1, push with c_x = -1), cell 1 at x = nx - 1 reaches
  // x = nx at x = 0 (pull with c_x = -1, push with c_x = +1).
  S* const Ai = A + i0;
  S* const A0 = Ai + (x0 == 0 ? (long long)g.nx : 0);
  S* const A1 = Ai + 1 - (x0 + 1 == g.nx - 1 ? (long long)g.nx : 0);
  // read / write / own slot of direction d relative to a row base
  const auto rd = [&](S* b, int d) { return b + p.off_rd[d]; };
  const auto wr = [&](S* b, int d) { return b + p.off_wr[d]; };
  const auto own = [&](S* b, int d) { return b + (long long)d * g.plane; };
  C f0[Q], f1[Q];
  if (coord_fast) {
#pragma unroll
    for (int d = 0; d < Q; d++) {
      if (cx(d) == 0) {
        Pair2<S>::ld(rd(Ai, d), f0[d], f1[d]);
      } else if (cx(d) == 1) {
        f0[d] = ld_fast<SP>(rd(A0, d), d, C(p.rho0));
        f1[d] = ld_fast<SP>(rd(Ai, d) + 1, d, C(p.rho0));
      } else {
        f0[d] = ld_fast<SP>(rd(Ai, d), d, C(p.rho0));
        f1[d] = ld_fast<SP>(rd(A1, d), d, C(p.rho0));
      }
    }
  }
  const bool solid0 = (fl0 & F_SOLID) != 0, solid1 = (fl1 & F_SOLID) != 0;
  uint32_t bc0 = 0, bc1 = 0;
  bool st0 = true, st1 = true;
  if (!solid0 && (fl0 & F_NEAR)) {
    const unsigned long long lw = p.links[i0];
    bc0 = (uint32_t)(lw & 0x3FFFFu);
    st0 = bc0 == (uint32_t)((lw >> 18) & 0x3FFFFu) && ((lw >> 36) & 0x3FFFFu) == 0 && !(fl0 & F_SOLID_PREV);
  }
  if (!solid1 && (fl1 & F_NEAR)) {
    const unsigned long long lw = p.links[i0 + 1];
    bc1 = (uint32_t)(lw & 0x3FFFFu);
    st1 = bc1 == (uint32_t)((lw >> 18) & 0x3FFFFu) && ((lw >> 36) & 0x3FFFFu) == 0 && !(fl1 & F_SOLID_PREV);
  }
  const bool both_solid = solid0 && solid1;
  const bool fast = coord_fast && st0 && st1;
  if (__all_sync(0xffffffffu, both_solid || fast)) {
    if (!both_solid) {
      if (bc0 | bc1) {  // bounce-back values are kept in the own slots
#pragma unroll
        for (int d = 0; d < 18; d++) {
          if ((bc0 >> d) & 1u) f0[d] = ld_fast<SP>(own(Ai, d), d, C(p.rho0));
          if ((bc1 >> d) & 1u) f1[d] = ld_fast<SP>(own(Ai, d) + 1, d, C(p.rho0));
        }
      }
      const bool plain = !solid0 && !solid1 && !(bc0 | bc1);
      const C rho0 = C(p.rho0);
      C p0[Q];
      if (!solid0) {
        pair_cell<SP, true, TRT, FORCE>(p, f0, p0);
      } else {
#pragma unroll
        for (int d = 0; d < Q; d++) p0[d] = C(0);
      }
      if (plain) {  // x-shifted directions of cell 0 (the others pair below)
#pragma unroll
        for (int j = 0; j < Q; j++)
          if (cx(j) != 0) st_fast<SP>(wr(cx(j) == 1 ? Ai : A0, j), p0[j], j, rho0);
      } else if (!solid0) {
#pragma unroll
        for (int j = 0; j < Q; j++) {
          const int oj = opp(j);
          S* a = wr(cx(j) == -1 ? A0 : Ai, j);
          if (j < 18 && ((bc0 >> oj) & 1u)) a = own(Ai, oj);
          st_fast<SP>(a, p0[j], j, rho0);
        }
      }
      if (p.compute_force && bc0) {
        pair_links<SP>(p, x0, y, z, bc0, p0, acc);
        has_link = true;
      }
      C p1[Q];
      if (!solid1) {
        pair_cell<SP, true, TRT, FORCE>(p, f1, p1);
      } else {
#pragma unroll
        for (int d = 0; d < Q; d++) p1[d] = C(0);
      }
      if (plain) {
#pragma unroll
        for (int j = 0; j < Q; j++) {
          if (cx(j) == 0)
            Pair2<S>::st(wr(Ai, j), p0[j], p1[j]);
          else
            st_fast<SP>(cx(j) == 1 ? wr(A1, j) : wr(Ai, j) + 1, p1[j], j, rho0);
        }
      } else if (!solid1) {
#pragma unroll
        for (int j = 0; j < Q; j++) {
          const int oj = opp(j);
          S* a = cx(j) == 1 ? wr(A1, j) : wr(Ai, j) + 1;
          if (j < 18 && ((bc1 >> oj) & 1u)) a = own(Ai, oj) + 1;
          st_fast<SP>(a, p1[j], j, rho0);
        }
      }
      if (p.compute_force && bc1) {
        pair_links<SP>(p, x0 + 1, y, z, bc1, p1, acc);
        has_link = true;
      }
    }
  } else {
    if (inb && !solid0) aa_general<SP, true, TRT, FORCE>(p, A, flags, x0, y, z, i0, (uint8_t)fl0, acc, &has_link);
    if (inb && !solid1) aa_general<SP, true, TRT, FORCE>(p, A, flags, x0 + 1, y, z, i0 + 1, (uint8_t)fl1, acc, &has_link);
  }
}

template <class SP, bool TRT, int FORCE>
__global__ void __launch_bounds__(256, (SP::MIN_BLOCKS > 2 ? 3 : 1)) aa_pair_split_kernel(const __grid_constant__ AAParams p,
                                                                                typename SP::S* __restrict__ A,
                                                                                const uint8_t* __restrict__ flags) {
  const Grid& g = p.g;
  const int x0 = 2 * (blockIdx.x * blockDim.x + threadIdx.x);
  const int y = blockIdx.y * blockDim.y + threadIdx.y;
  const int z = blockIdx.z;
  const bool inb = x0 < g.nx && y < g.ny;
  clear_record(p.zero_next);
  if (ghost_plane(p, z)) return;  // whole block in a ghost plane
  double acc[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
  bool has_link = false;
  pair_split_cells<SP, TRT, FORCE>(p, A, flags, x0, y, z, inb, acc, has_link);
  if (p.compute_force) block_force_reduce(acc, has_link, p.force + block_stripe());
}


// ---- quad kernel: even phase, FP16-deviation storage ----------------------------------
// One thread updates four x-adjacent cells (x0 .. x0+3, x0 a multiple of 4).  In the even
// phase every direction reads and writes the cells' own slots, for four cells one aligned
// 8-byte word: 19 loads and 19 stores per four cells, addressing and control shared by
// four cells.  The cells collide in pairs, from the low and the high half2 of each word,
// and pack back to half2 at once, which bounds the live registers.
template <bool TRT, int FORCE>
__global__ void __launch_bounds__(256, 2) aa_quad_even_kernel(const __grid_constant__ AAParams p,
                                                              __half* __restrict__ A,
                                                              const uint8_t* __restrict__ flags) {
  using SP = StF16;
  using C = float;
  const Grid& g = p.g;
  const int x0 = 4 * (blockIdx.x * blockDim.x + threadIdx.x);
  const int y = blockIdx.y * blockDim.y + threadIdx.y;
  const int z = blockIdx.z;
  const bool inb = x0 < g.nx && y < g.ny;
  clear_record(p.zero_next);
  if (ghost_plane(p, z)) return;  // whole block in a ghost plane
  double acc[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
  bool has_link = false;
  const long long i0 = inb ? node_index(g, x0, y, z) : 0;
  uint32_t fw = 0x01010101u * F_SOLID;
  if (inb) fw = *reinterpret_cast<const uint32_t*>(flags + i0);
  __half* const Ai = A + i0;
  uint2 w[Q];
  if (inb) {
#pragma unroll
    for (int d = 0; d < Q; d++)  // byte offsets: one 64-bit add per access (-2 % on B200)
      w[d] = *reinterpret_cast<const uint2*>(reinterpret_cast<const char*>(Ai) + p.offb_rd[d]);
  }
  uint32_t bc[4];
  bool fast = true, any_fluid = false;
#pragma unroll
  for (int k = 0; k < 4; k++) {
    const uint32_t fl = (fw >> (8 * k)) & 0xFFu;
    bc[k] = 0;
    if (!(fl & F_SOLID)) {
      any_fluid = true;
      if (fl & F_NEAR) {
        const unsigned long long lw = p.links[i0 + k];
        bc[k] = (uint32_t)(lw & 0x3FFFFu);
        fast = fast && bc[k] == (uint32_t)((lw >> 18) & 0x3FFFFu) && ((lw >> 36) & 0x3FFFFu) == 0 &&
               !(fl & F_SOLID_PREV);
      }
    }
  }
  if (__all_sync(0xffffffffu, !any_fluid || fast)) {
    if (any_fluid) {
      uint32_t out[2][Q];
#pragma unroll
      for (int h = 0; h < 2; h++) {
        const int ka = 2 * h, kb = 2 * h + 1;
        C pa[Q], pb[Q];
        {
          C f[Q];
#pragma unroll
          for (int d = 0; d < Q; d++) {
            const uint32_t u = h ? w[d].y : w[d].x;
            f[d] = __low2float(*reinterpret_cast<const __half2*>(&u));
          }
          if (!((fw >> (8 * ka)) & F_SOLID)) {
            pair_cell<SP, false, TRT, FORCE>(p, f, pa);
          } else {
#pragma unroll
            for (int d = 0; d < Q; d++) pa[d] = C(0);
          }
        }
        {
          C f[Q];
#pragma unroll
          for (int d = 0; d < Q; d++) {
            const uint32_t u = h ? w[d].y : w[d].x;
            f[d] = __high2float(*reinterpret_cast<const __half2*>(&u));
          }
          if (!((fw >> (8 * kb)) & F_SOLID)) {
            pair_cell<SP, false, TRT, FORCE>(p, f, pb);
          } else {
#pragma unroll
            for (int d = 0; d < Q; d++) pb[d] = C(0);
          }
        }
#pragma unroll
        for (int j = 0; j < Q; j++) {  // own slot j takes the post-collision value of opp(j)
          const __half2 v = __floats2half2_rn(pa[opp(j)], pb[opp(j)]);
          out[h][j] = *reinterpret_cast<const uint32_t*>(&v);
        }
        if (p.compute_force && (bc[ka] | bc[kb])) {
          pair_links<SP>(p, x0 + ka, y, z, bc[ka], pa, acc);
          pair_links<SP>(p, x0 + kb, y, z, bc[kb], pb, acc);
          has_link = true;
        }
      }
#pragma unroll
      for (int j = 0; j < Q; j++)
        *reinterpret_cast<uint2*>(reinterpret_cast<char*>(Ai) + p.offb_wr[j]) = make_uint2(out[0][j], out[1][j]);
    }
  } else {
#pragma unroll 1
    for (int k = 0; k < 4; k++) {
      const uint32_t fl = (fw >> (8 * k)) & 0xFFu;
      if (inb && !(fl & F_SOLID))
        aa_general<SP, false, TRT, FORCE>(p, A, flags, x0 + k, y, z, i0 + k, (uint8_t)fl, acc, &has_link);
    }
  }
  if (p.compute_force) block_force_reduce(acc, has_link, p.force + block_stripe());
}

// ---- octo kernel: even phase, FP16-deviation storage -----------------------------------
// Eight x-adjacent cells per thread (x0 a multiple of 8): one aligned 16-byte word per
// direction, 19 loads and 19 stores of 128 bits for eight cells.  The cells collide in pairs
// (the four half2 lanes of the words); each pair's results replace that pair's lane of the
// words at once (its inputs are consumed by then), so the words hold inputs and outputs
// without a second set of registers.
__device__ __forceinline__ uint32_t u4get(const uint4& v, const int k) {
  return k == 0 ? v.x : (k == 1 ? v.y : (k == 2 ? v.z : v.w));
}
__device__ __forceinline__ void u4set(uint4& v, const int k, const uint32_t u) {
  if (k == 0) v.x = u;
  else if (k == 1) v.y = u;
  else if (k == 2) v.z = u;
  else v.w = u;
}

template <bool TRT, int FORCE>
__global__ void __launch_bounds__(128, 3) aa_octo_even_kernel(const __grid_constant__ AAParams p,
                                                              __half* __restrict__ A,
                                                              const uint8_t* __restrict__ flags) {
  using SP = StF16;
  using C = float;
  const Grid& g = p.g;
  const int x0 = 8 * (blockIdx.x * blockDim.x + threadIdx.x);
  const int y = blockIdx.y * blockDim.y + threadIdx.y;
  const int z = blockIdx.z;
  const bool inb = x0 < g.nx && y < g.ny;
  clear_record(p.zero_next);
  if (ghost_plane(p, z)) return;  // whole block in a ghost plane
  double acc[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
  bool has_link = false;
  const long long i0 = inb ? node_index(g, x0, y, z) : 0;
  uint2 fw = make_uint2(0x01010101u * F_SOLID, 0x01010101u * F_SOLID);
  if (inb) fw = *reinterpret_cast<const uint2*>(flags + i0);
  char* const Ai = reinterpret_cast<char*>(A + i0);
  uint4 w[Q];
  if (inb) {
#pragma unroll
    for (int d = 0; d < Q; d++) w[d] = *reinterpret_cast<const uint4*>(Ai + p.offb_rd[d]);
  }
  bool fast = true, any_fluid = false;
#pragma unroll
  for (int k = 0; k < 8; k++) {
    const uint32_t fl = ((k < 4 ? fw.x : fw.y) >> (8 * (k & 3))) & 0xFFu;
    if (!(fl & F_SOLID)) {
      any_fluid = true;
      if (fl & F_NEAR) {
        const unsigned long long lw = p.links[i0 + k];
        const uint32_t b = (uint32_t)(lw & 0x3FFFFu);
        fast = fast && b == (uint32_t)((lw >> 18) & 0x3FFFFu) && ((lw >> 36) & 0x3FFFFu) == 0 && !(fl & F_SOLID_PREV);
      }
    }
  }
  if (__all_sync(0xffffffffu, !any_fluid || fast)) {
    if (any_fluid) {
#pragma unroll
      for (int h = 0; h < 4; h++) {
        const int ka = 2 * h, kb = 2 * h + 1;
        const uint32_t fla = ((h < 2 ? fw.x : fw.y) >> (16 * (h & 1))) & 0xFFu;
        const uint32_t flb = ((h < 2 ? fw.x : fw.y) >> (16 * (h & 1) + 8)) & 0xFFu;
        C pa[Q], pb[Q];
        {
          C f[Q];
#pragma unroll
          for (int d = 0; d < Q; d++) {
            const uint32_t u = u4get(w[d], h);
            f[d] = __low2float(*reinterpret_cast<const __half2*>(&u));
          }
          if (!(fla & F_SOLID)) {
            pair_cell<SP, false, TRT, FORCE>(p, f, pa);
          } else {
#pragma unroll
            for (int d = 0; d < Q; d++) pa[d] = C(0);
          }
        }
        {
          C f[Q];
#pragma unroll
          for (int d = 0; d < Q; d++) {
            const uint32_t u = u4get(w[d], h);
            f[d] = __high2float(*reinterpret_cast<const __half2*>(&u));
          }
          if (!(flb & F_SOLID)) {
            pair_cell<SP, false, TRT, FORCE>(p, f, pb);
          } else {
#pragma unroll
            for (int d = 0; d < Q; d++) pb[d] = C(0);
          }
        }
#pragma unroll
        for (int j = 0; j < Q; j++) {  // own slot j takes the post-collision value of opp(j)
          const __half2 v = __floats2half2_rn(pa[opp(j)], pb[opp(j)]);
          u4set(w[j], h, *reinterpret_cast<const uint32_t*>(&v));
        }
        if (p.compute_force && ((fla | flb) & F_NEAR)) {
          const unsigned long long la = (fla & F_NEAR) ? p.links[i0 + ka] : 0ull;
          const unsigned long long lb = (flb & F_NEAR) ? p.links[i0 + kb] : 0ull;
          pair_links<SP>(p, x0 + ka, y, z, (uint32_t)(la & 0x3FFFFu), pa, acc);
          pair_links<SP>(p, x0 + kb, y, z, (uint32_t)(lb & 0x3FFFFu), pb, acc);
          has_link = has_link || ((la | lb) & 0x3FFFFu) != 0;
        }
      }
#pragma unroll
      for (int j = 0; j < Q; j++) *reinterpret_cast<uint4*>(Ai + p.offb_wr[j]) = w[j];
    }
  } else {
#pragma unroll 1
    for (int k = 0; k < 8; k++) {
      const uint32_t fl = ((k < 4 ? fw.x : fw.y) >> (8 * (k & 3))) & 0xFFu;
      if (inb && !(fl & F_SOLID))
        aa_general<SP, false, TRT, FORCE>(p, A, flags, x0 + k, y, z, i0 + k, (uint8_t)fl, acc, &has_link);
    }
  }
  if (p.compute_force) block_force_reduce(acc, has_link, p.force + block_stripe());
}

// Ordinal (0..9) of an x-shifted D3Q19 direction among the ten.
__host__ __device__ constexpr int xslot(int d) {
  int n = 0;
  for (int e = 0; e < d; e++) n += cx(e) != 0 ? 1 : 0;
  return n;
}

// The split pair update of `pairs` cell pairs from x0 (blocks off the word path); out of
// line, which keeps the word path's code compact.
template <bool TRT, int FORCE>
__device__ __noinline__ void odd_pairs_fallback(const AAParams& p, __half* __restrict__ A,
                                                const uint8_t* __restrict__ flags, const int x0, const int pairs,
                                                const int y, const int z, const bool inb, double* acc, bool* has_out) {
  bool has_link = *has_out;
#pragma unroll 1
  for (int h = 0; h < pairs; h++) pair_split_cells<StF16, TRT, FORCE>(p, A, flags, x0 + 2 * h, y, z, inb, acc, has_link);
  *has_out = has_link;
}

// Stores the elements of an 8-byte word whose bit in `skip` is clear (2-byte elements; q
// 8-byte aligned).
__device__ __forceinline__ void st_u2_masked(char* q, const uint2 v, const uint32_t skip) {
#pragma unroll
  for (int k = 0; k < 4; k++)
    if (!((skip >> k) & 1u))
      *reinterpret_cast<unsigned short*>(q + 2 * k) = (unsigned short)((k < 2 ? v.x : v.y) >> (16 * (k & 1)));
}

// ---- quad kernel: odd phase, FP16-deviation storage ----------------------------------
// One block holds whole rows: nx / 4 threads per row (nx a multiple of 128, at most 1024),
// four x-adjacent cells per thread (x0 a multiple of 4), at most 256 threads.  Every
// direction moves as one aligned 8-byte word per thread: for an x-shifted direction the word
// of the thread's own four positions is shifted by one element, and the element that enters
// comes from the neighbouring thread of the row through shared memory (the last thread of a
// row neighbours the first: periodic x); every thread takes part, so the exchange has no
// divergent branch.  The outputs are shifted back the same way before the 19 word stores.
// Solid cells are collided with whatever their slots hold and left out when the words are
// stored: a word that carries a solid cell's output is stored element by element without
// it, because that element would land on the own slot where the fluid neighbour keeps its
// bounce-back value.  Fluid cells next to a solid (static links) stay on the word path:
// they take their bounce-back inputs from their own slots and write the outputs that point
// into a solid to their own slots; the word elements they push into a solid node's slot
// are dead (no cell reads them while the node is solid).  Every other slot is read and
// written by exactly the thread of the cell whose pull/push set holds it.  Blocks holding a
// cell with a moving or changed link, an uncovered cell, or a row next to a y/z wrap (or
// past ny) run the split pair update instead (block vote).
template <bool TRT, int FORCE>
__global__ void __launch_bounds__(256, 2) aa_quad_odd_kernel(const __grid_constant__ AAParams p,
                                                             __half* __restrict__ A,
                                                             const uint8_t* __restrict__ flags) {
  using SP = StF16;
  using C = float;
  const Grid& g = p.g;
  // this thread and its x neighbours in the row (periodic) in the exchange arrays
  const int nxt = (int)blockDim.x;  // threads per row
  const int tid = (int)threadIdx.x + nxt * (int)threadIdx.y;
  const int tprev = tid + ((int)threadIdx.x == 0 ? nxt - 1 : -1);
  const int tnext = tid + ((int)threadIdx.x == nxt - 1 ? 1 - nxt : 1);
  const int x0 = 4 * (int)threadIdx.x;
  const int y = blockIdx.y * blockDim.y + threadIdx.y;
  const int z = blockIdx.z;
  const bool inb = y < g.ny;
  clear_record(p.zero_next);
  if (ghost_plane(p, z)) return;  // whole block in a ghost plane
  // exchange: the element of each x-shifted direction (slot xslot(d)) that enters the
  // neighbouring thread's word, and the solid masks
  __shared__ unsigned short xin[10][256], xout[10][256];
  __shared__ unsigned char xsk[256];
  double acc[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
  bool has_link = false;
  const long long i0 = inb ? node_index(g, x0, y, z) : 0;
  uint32_t fw = 0x01010101u * F_SOLID;
  if (inb) fw = *reinterpret_cast<const uint32_t*>(flags + i0);
  uint32_t smask = 0;  // bit k: cell x0 + k is solid
  bool fast = inb && y > 0 && y < g.ny - 1 && z > 0 && z < g.nz - 1;
#pragma unroll
  for (int k = 0; k < 4; k++) {
    const uint32_t fl = (fw >> (8 * k)) & 0xFFu;
    if (fl & F_SOLID) {
      smask |= 1u << k;
    } else {
      if (fl & F_SOLID_PREV) fast = false;
      if (fl & F_NEAR) {
        const unsigned long long lw = p.links[i0 + k];
        fast = fast && (uint32_t)(lw & 0x3FFFFu) == (uint32_t)((lw >> 18) & 0x3FFFFu) && ((lw >> 36) & 0x3FFFFu) == 0;
      }
    }
  }
  if (__syncthreads_and(fast)) {
    char* const Ai = reinterpret_cast<char*>(A + i0);
    const C rho0 = C(p.rho0);
    uint2 w[Q];
#pragma unroll
    for (int d = 0; d < Q; d++) {
      // offb_rd addresses element x0 - c_dx of the source row: the aligned word is at x0
      w[d] = *reinterpret_cast<const uint2*>(Ai + p.offb_rd[d] + 2 * cx(d));
    }
#pragma unroll
    for (int d = 0; d < Q; d++) {
      if (cx(d) == 1) xin[xslot(d)][tid] = (unsigned short)(w[d].y >> 16);      // last element
      if (cx(d) == -1) xin[xslot(d)][tid] = (unsigned short)(w[d].x & 0xFFFFu);  // first element
    }
    xsk[tid] = (unsigned char)smask;
    __syncthreads();
    // shift the x-pulled words by one element (element k = bits 16(k%2) of 32-bit word k/2)
#pragma unroll
    for (int d = 0; d < Q; d++) {
      const uint2 v = w[d];
      if (cx(d) == 1) {  // [x0-1 .. x0+2]: the last element of the previous thread's word
        const uint32_t in = xin[xslot(d)][tprev];
        w[d] = make_uint2((v.x << 16) | in, __funnelshift_l(v.x, v.y, 16));
      } else if (cx(d) == -1) {  // [x0+1 .. x0+4]: the first element of the next thread's word
        const uint32_t in = xin[xslot(d)][tnext];
        w[d] = make_uint2(__funnelshift_r(v.x, v.y, 16), (v.y >> 16) | (in << 16));
      }
    }
    // collide the cells in pairs (low and high half2 of each 32-bit word); each pair's
    // outputs replace its inputs in the words.  Solid cells compute values that are never
    // stored.
#pragma unroll
    for (int h = 0; h < 2; h++) {
      const int ka = 2 * h, kb = 2 * h + 1;
      const uint32_t fla = (fw >> (16 * h)) & 0xFFu, flb = (fw >> (16 * h + 8)) & 0xFFu;
      const uint32_t bca = (fla & F_NEAR) && !(fla & F_SOLID) ? (uint32_t)(p.links[i0 + ka] & 0x3FFFFu) : 0u;
      const uint32_t bcb = (flb & F_NEAR) && !(flb & F_SOLID) ? (uint32_t)(p.links[i0 + kb] & 0x3FFFFu) : 0u;
      C pa[Q], pb[Q];
      {
        C f[Q];
#pragma unroll
        for (int d = 0; d < Q; d++) {
          const uint32_t u = h ? w[d].y : w[d].x;
          f[d] = __low2float(*reinterpret_cast<const __half2*>(&u));
        }
        if (bca) {  // bounce-back values are kept in the own slots
#pragma unroll
          for (int d = 0; d < 18; d++)
            if ((bca >> d) & 1u) f[d] = ld_fast<SP>(A + (long long)d * g.plane + i0 + ka, d, rho0);
        }
        pair_cell<SP, true, TRT, FORCE>(p, f, pa);
      }
      {
        C f[Q];
#pragma unroll
        for (int d = 0; d < Q; d++) {
          const uint32_t u = h ? w[d].y : w[d].x;
          f[d] = __high2float(*reinterpret_cast<const __half2*>(&u));
        }
        if (bcb) {
#pragma unroll
          for (int d = 0; d < 18; d++)
            if ((bcb >> d) & 1u) f[d] = ld_fast<SP>(A + (long long)d * g.plane + i0 + kb, d, rho0);
        }
        pair_cell<SP, true, TRT, FORCE>(p, f, pb);
      }
#pragma unroll
      for (int j = 0; j < Q; j++) {  // push slot j takes the post-collision value of j
        const __half2 v = __floats2half2_rn(pa[j], pb[j]);
        const uint32_t u = *reinterpret_cast<const uint32_t*>(&v);
        if (h)
          w[j].y = u;
        else
          w[j].x = u;
      }
      if (bca | bcb) {  // outputs into a solid go to the own slots
#pragma unroll
        for (int j = 0; j < 18; j++) {
          const int oj = opp(j);
          if ((bca >> oj) & 1u) st_fast<SP>(A + (long long)oj * g.plane + i0 + ka, pa[j], j, rho0);
          if ((bcb >> oj) & 1u) st_fast<SP>(A + (long long)oj * g.plane + i0 + kb, pb[j], j, rho0);
        }
        if (p.compute_force) {
          pair_links<SP>(p, x0 + ka, y, z, bca, pa, acc);
          pair_links<SP>(p, x0 + kb, y, z, bcb, pb, acc);
          has_link = true;
        }
      }
    }
#pragma unroll
    for (int j = 0; j < Q; j++) {
      if (cx(j) == 1) xout[xslot(j)][tid] = (unsigned short)(w[j].y >> 16);      // the fourth cell's output
      if (cx(j) == -1) xout[xslot(j)][tid] = (unsigned short)(w[j].x & 0xFFFFu);  // the first cell's output
    }
    __syncthreads();
    // solid cells among the six whose outputs the stored words carry: bit 0 = cell x0 - 1,
    // bits 1..4 = cells x0 .. x0+3, bit 5 = cell x0 + 4
    const uint32_t win = (((uint32_t)xsk[tprev] >> 3) & 1u) | (smask << 1) | (((uint32_t)xsk[tnext] & 1u) << 5);
#pragma unroll
    for (int j = 0; j < Q; j++) {
      const uint2 v = w[j];
      uint2 nw = v;
      uint32_t skip = (win >> 1) & 0xFu;  // cells x0 .. x0+3
      if (cx(j) == 1) {  // push to x + 1: the word at x0 carries cells x0-1 .. x0+2
        const uint32_t in = xout[xslot(j)][tprev];
        nw = make_uint2((v.x << 16) | in, __funnelshift_l(v.x, v.y, 16));
        skip = win & 0xFu;
      } else if (cx(j) == -1) {  // push to x - 1: the word at x0 carries cells x0+1 .. x0+4
        const uint32_t in = xout[xslot(j)][tnext];
        nw = make_uint2(__funnelshift_r(v.x, v.y, 16), (v.y >> 16) | (in << 16));
        skip = (win >> 2) & 0xFu;
      }
      // offb_wr addresses element x0 + c_jx of the target row: the aligned word is at x0
      char* const q = Ai + p.offb_wr[j] - 2 * cx(j);
      if (skip == 0u)
        *reinterpret_cast<uint2*>(q) = nw;
      else
        st_u2_masked(q, nw, skip);
    }
  } else {
    odd_pairs_fallback<TRT, FORCE>(p, A, flags, x0, 2, y, z, inb, acc, &has_link);
  }
  if (p.compute_force) block_force_reduce(acc, has_link, p.force + block_stripe());
}

// q = n / d and r = n % d for n < 2^31 through an FP64 reciprocal (exact after the
// one-step correction; the product is off by at most one).
__device__ __forceinline__ void divmod_rcp(const unsigned n, const int d, const double inv, unsigned& q, int& r) {
  q = (unsigned)((double)n * inv);
  r = (int)(n - q * (unsigned)d);
  if (r < 0) {
    q--;
    r += d;
  } else if (r >= d) {
    q++;
    r -= d;
  }
}


// ---- batched persistent step over many domains -------------------------------------
// Work items are runs of BATCH_ITEM consecutive cells of one domain; every domain's
// items are numbered consecutively and item_dom maps an item to its domain.  Each
// block takes one contiguous range of items (equal counts +-1), so the domain, and
// with it the parameter block copied to shared memory, changes rarely.  The phase
// and the force record of a domain follow from the device step counter, which a
// one-thread kernel advances after every step: the same launch sequence can be
// captured once in a CUDA graph and replayed.
// One kernel per phase: the ODD instance updates the domains whose phase this step is
// odd and skips the others (both are launched every step), so each holds one phase's
// code.
template <class SP, bool ODD, bool TRT, int FORCE, bool FACES>
__global__ void __launch_bounds__(BATCH_ITEM, LBM_BATCH_MINB(SP)) aa_batch_kernel(const __grid_constant__ BatchParams bp) {
  __shared__ AAParams sp;
  using S = typename SP::S;
  const int t = threadIdx.x;
  const long long k = *bp.counter;
  const long long G = gridDim.x;
  const long long first = bp.items * blockIdx.x / G, last = bp.items * (blockIdx.x + 1) / G;
  int dom = -1;
  S* A = nullptr;
  const uint8_t* flags = nullptr;
  double* rec = nullptr;
  long long item0 = 0;
  double inv_nx = 0.0, inv_ny = 0.0;
  // force / torque of the current domain, reduced once per domain and block
  double acc[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
  bool has_link = false;
  const int stripe = (int)(blockIdx.x % FORCE_SLOTS) * 8;
  for (long long item = first; item < last; item++) {
    const int d = bp.item_dom[item];
    if (d != dom) {
      const BatchDom& D = bp.doms[d];
      if ((int)((D.phase0 + k) & 1) != (ODD ? 1 : 0)) {  // the other phase's kernel takes it
        item = D.item_end - 1;
        continue;
      }
      if (dom >= 0 && sp.compute_force) {
        block_force_reduce(acc, has_link, rec + stripe);
#pragma unroll
        for (int c = 0; c < 6; c++) acc[c] = 0.0;
        has_link = false;
      }
      __syncthreads();  // every thread is done with the previous parameter block
      dom = d;
      const int* src = reinterpret_cast<const int*>(&D.p[ODD ? 1 : 0]);
      int* dst = reinterpret_cast<int*>(&sp);
      for (int w = t; w < (int)(sizeof(AAParams) / sizeof(int)); w += BATCH_ITEM) dst[w] = src[w];
      A = (S*)D.A;
      flags = D.flags;
      const long long step = D.base_step + k + 1;  // the domain's step being computed
      rec = D.ring + (size_t)(step % D.ring_slots) * FORCE_RECORD;
      item0 = D.item_begin;
      if (item == item0) {  // this block holds the domain's first item: clear the next record
        double* next = D.ring + (size_t)((step + 1) % D.ring_slots) * FORCE_RECORD;
        for (int w = t; w < FORCE_RECORD; w += BATCH_ITEM) next[w] = 0.0;
      }
      __syncthreads();
      inv_nx = 1.0 / (double)sp.g.nx;
      inv_ny = 1.0 / (double)sp.g.ny;
    }
    const Grid& g = sp.g;
    // a domain holds fewer than 2^31 cells: 32-bit index arithmetic.  Cells keep the
    // row order (x fastest): ordering the x-face columns apart made their warps read
    // 19 x 32 separate sectors (stride nx) and was slower overall.
    const unsigned cell = (unsigned)(item - item0) * BATCH_ITEM + t;
    const bool inb = cell < (unsigned)g.N;
    unsigned row, z;
    int x, y;
    divmod_rcp(cell, g.nx, inv_nx, row, x);
    divmod_rcp(row, g.ny, inv_ny, z, y);
    aa_direct<GlobalSpace<SP>, ODD, TRT, FORCE, FACES>(sp, A, flags, x, y, (int)z, inb, acc, &has_link);
  }
  if (dom >= 0 && sp.compute_force) block_force_reduce(acc, has_link, rec + stripe);
}

// ---- TMA-staged persistent step ------------------------------------------------------
// Tiles are row segments of TW cells.  For every tile without a boundary node, one
// thread streams the 19 direction segments it needs (even phase: the node's own
// slots; odd phase: the neighbour slots, row-shifted, plus a 16-byte halo for the
// x-shifted directions) into shared memory with cp.async.bulk, several tiles ahead,
// completion tracked by one mbarrier per stage.  The compute reads shared memory,
// so loads stay in flight while warps compute.  Tiles holding a boundary node are
// processed by the direct path.
__device__ __forceinline__ uint32_t smem_u32(const void* ptr) {
  return (uint32_t)__cvta_generic_to_shared(ptr);
}
__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint32_t bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}
__device__ __forceinline__ void bulk_g2s(uint32_t dst, const void* src, uint32_t bytes, uint32_t bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(dst),
               "l"(src), "r"(bytes), "r"(bar)
               : "memory");
}
// Bounded wait on an mbarrier phase: gives up after `polls` polls (default ~2^22; each
// try_wait blocks for a hardware-defined interval), returning false.
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity, int polls = MBAR_WAIT_POLLS) {
  for (int it = 0; it < polls; it++) {
    uint32_t ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(bar), "r"(parity)
        : "memory");
    if (ok) return true;
  }
  return false;
}

// Probe of the bounded wait above: thread 0 initialises an mbarrier that expects one
// arrival, nothing arrives and no copy targets it, so every thread's wait gives up after
// `polls` polls; the block then records the failure in *err as the step kernels do.
// Nothing is in flight when the kernel returns.
static __global__ void __launch_bounds__(32) wait_probe_kernel(const int polls, int* err) {
  __shared__ __align__(8) unsigned long long bar;
  if (threadIdx.x == 0) {
    mbar_init(smem_u32(&bar), 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();
  const bool ok = mbar_wait(smem_u32(&bar), 0u, polls);
  if (!__all_sync(0xffffffffu, ok) && threadIdx.x == 0) atomicExch(err, 1);
}

constexpr int TMA_MAX_STAGES = 8;

template <class SP, bool ODD>
__device__ __forceinline__ void tma_issue(const AAParams& p, const typename SP::S* A, long long tile,
                                          unsigned char* stage, uint32_t bar) {
  using S = typename SP::S;
  const Grid& g = p.g;
  const TmaCfg& T = p.tma;
  const int tw = T.tw, H = T.halo;
  const long long row = tile / T.ntx;
  const int x0 = (int)(tile - row * T.ntx) * tw;
  const int y = (int)(row % g.ny), z = (int)(row / g.ny);
  const uint32_t seg = (uint32_t)(tw * sizeof(S)), hal = 16u;
  mbar_expect_tx(bar, ODD ? 19u * seg + 10u * hal : 19u * seg);
  const uint32_t dst0 = smem_u32(stage);
  const uint32_t dstride = (uint32_t)(T.buf_elems * sizeof(S));
#pragma unroll 1
  for (int d = 0; d < Q; d++) {
    const uint32_t dst = dst0 + d * dstride;
    if (!ODD) {
      bulk_g2s(dst, A + (long long)d * g.plane + row * g.nx + x0, seg, bar);
      continue;
    }
    int ys = y - cy(d), zs = z - cz(d);
    ys = ys < 0 ? ys + g.ny : (ys >= g.ny ? ys - g.ny : ys);
    zs = zs < 0 ? zs + g.nz : (zs >= g.nz ? zs - g.nz : zs);
    const S* rowp = A + (long long)opp(d) * g.plane + ((long long)zs * g.ny + ys) * g.nx;
    const int c = cx(d);
    if (c == 0) {
      bulk_g2s(dst, rowp + x0, seg, bar);
    } else if (c == 1) {  // source x-1: [halo | main]
      bulk_g2s(dst, rowp + (x0 >= H ? x0 - H : g.nx - H), hal, bar);
      bulk_g2s(dst + hal, rowp + x0, seg, bar);
    } else {  // source x+1: [main | halo]
      bulk_g2s(dst, rowp + x0, seg, bar);
      bulk_g2s(dst + seg, rowp + (x0 + tw < g.nx ? x0 + tw : 0), hal, bar);
    }
  }
}

template <class SP, bool ODD, bool TRT, int FORCE>
__global__ void __launch_bounds__(128) aa_tma_kernel(const __grid_constant__ AAParams p,
                                                     typename SP::S* __restrict__ A,
                                                     const uint8_t* __restrict__ flags) {
  using S = typename SP::S;
  using C = typename SP::C;
  extern __shared__ __align__(128) unsigned char smem[];
  __shared__ __align__(8) unsigned long long bars[TMA_MAX_STAGES];
  const Grid& g = p.g;
  const TmaCfg& T = p.tma;
  const int t = threadIdx.x;
  const int NS = T.stages;
  const long long G = gridDim.x;
  const long long first = blockIdx.x;
  const long long ntb = first < T.ntiles ? (T.ntiles - first + G - 1) / G : 0;
  const uint8_t slow_bit = ODD ? 2 : 1;
  clear_record(p.zero_next);
  if (t == 0) {
    for (int s = 0; s < NS; s++) mbar_init(smem_u32(&bars[s]), 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();
  uint32_t pending = 0;  // thread 0: stages with loads in flight
  auto issue = [&](long long k) {
    if (k >= ntb) return;
    const long long tile = first + k * G;
    if (T.tile_slow[tile] & slow_bit) return;
    const int s = (int)(k % NS);
    tma_issue<SP, ODD>(p, A, tile, smem + (size_t)s * T.stage_bytes, smem_u32(&bars[s]));
    pending |= 1u << s;
  };
  if (t == 0)
    for (long long k = 0; k < NS - 1; k++) issue(k);
  uint32_t phases = 0;
  double acc[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
  bool has_link = false;
  bool failed = false;
  const C rho0 = C(p.rho0);
  const Coll<C> kc{C(p.omega_p), C(p.omega_m), C(p.gacc[0]), C(p.gacc[1]), C(p.gacc[2])};
  for (long long k = 0; k < ntb; k++) {
    const long long tile = first + k * G;
    const int s = (int)(k % NS);
    if (t == 0) issue(k + NS - 1);
    const long long row = tile / T.ntx;
    const int x0 = (int)(tile - row * T.ntx) * T.tw;
    const int y = (int)(row % g.ny), z = (int)(row / g.ny);
    const int x = x0 + t;
    if (T.tile_slow[tile] & slow_bit) {
      aa_direct<SP, ODD, TRT, FORCE, false>(p, A, flags, x, y, z, true, acc, &has_link);
      continue;
    }
    const bool ok = mbar_wait(smem_u32(&bars[s]), (phases >> s) & 1u);
    phases ^= 1u << s;
    const S* st = (const S*)(smem + (size_t)s * T.stage_bytes);
    C f[Q];
#pragma unroll
    for (int d = 0; d < Q; d++) {
      int idx = t;
      if (ODD) idx = cx(d) == 1 ? T.halo - 1 + t : (cx(d) == -1 ? t + 1 : t);
      f[d] = ld_fast<SP>(st + d * T.buf_elems + idx, d, rho0);
    }
    if (t == 0) pending &= ~(1u << s);
    if (!__syncthreads_and(ok)) {  // stage consumed (or a wait gave up everywhere)
      failed = true;
      break;
    }
    C rho, ux, uy, uz;
    moments<C, FORCE, SP::DEV>(f, kc, rho, ux, uy, uz, rho0);
    C pst[Q];
    collide<C, TRT, FORCE, SP::DEV>(f, pst, kc, rho, ux, uy, uz, rho0);
    const long long i = row * g.nx + x;
    S* const base = A + i;
    long long fix_lo = 0, fix_hi = 0;
    if (ODD) {
      fix_lo = x == 0 ? (long long)g.nx : 0;
      fix_hi = x == g.nx - 1 ? (long long)g.nx : 0;
    }
#pragma unroll
    for (int j = 0; j < Q; j++) {
      long long o = p.off_wr[j];
      if (ODD) {
        if (cx(j) == 1) o -= fix_hi;
        if (cx(j) == -1) o += fix_lo;
      }
      st_fast<SP>(base + o, ODD ? pst[j] : pst[opp(j)], j, rho0);
    }
  }
  if (failed) {
    if (t == 0) {
      atomicExch(T.err, 1);
      // drain the copies this block still has in flight (bounded)
      for (int s = 0; s < NS; s++)
        if (pending & (1u << s)) mbar_wait(smem_u32(&bars[s]), (phases >> s) & 1u);
    }
    __syncthreads();
  }
  if (p.compute_force) block_force_reduce(acc, has_link, p.force + block_stripe());
}

// ---- state readout (populations, macros, mass, finiteness) ---------------------------
// Reconstructs S_n[d, x] from the current layout using the flag bit `solid_bit`
// (the flags of the last completed step).
template <class SP>
__device__ __forceinline__ void aa_read(const ReadParams& p, const typename SP::S* A, const uint8_t* flags,
                                        int x, int y, int z, long long i, typename SP::C* f) {
  using C = typename SP::C;
  const Grid& g = p.g;
  const C rho0 = C(p.rho0);
  if (!p.swapped) {
#pragma unroll
    for (int d = 0; d < Q; d++) f[d] = SP::ld(A + (long long)d * g.plane + i, d, rho0);
    return;
  }
  const long long nxl = g.nx, nxy = (long long)g.nx * g.ny;
  const int xs[3] = {x == 0 ? (g.per[0] ? g.nx - 1 : -1) : x - 1, x,
                     x == g.nx - 1 ? (g.per[0] ? 0 : -1) : x + 1};
  const int ys[3] = {y == 0 ? (g.per[1] ? g.ny - 1 : -1) : y - 1, y,
                     y == g.ny - 1 ? (g.per[1] ? 0 : -1) : y + 1};
  const int zs[3] = {z == 0 ? (g.per[2] ? g.nz - 1 : -1) : z - 1, z,
                     z == g.nz - 1 ? (g.per[2] ? 0 : -1) : z + 1};
#pragma unroll
  for (int d = 0; d < Q; d++) {
    long long a = (long long)d * g.plane + i;
    if (d != 18) {
      const int sx = xs[1 - cx(d)], sy = ys[1 - cy(d)], sz = zs[1 - cz(d)];
      if ((sx | sy | sz) >= 0) {
        const long long src = sx + nxl * sy + nxy * sz;
        if (!(flags[src] & p.solid_bit)) a = (long long)opp(d) * g.plane + src;
      }
    }
    f[d] = SP::ld(A + a, d, rho0);
  }
}

template <class SP>
__global__ void aa_export_kernel(const ReadParams p, const typename SP::S* __restrict__ A,
                                 const uint8_t* __restrict__ flags, ExportOut out) {
  using C = typename SP::C;
  const Grid& g = p.g;
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  const int y = blockIdx.y * blockDim.y + threadIdx.y;
  const int z = blockIdx.z;
  if (x >= g.nx || y >= g.ny) return;
  const long long i = node_index(g, x, y, z);
  C f[Q];
  const bool solid = (flags[i] & p.solid_bit) != 0;
  if (solid) {
#pragma unroll
    for (int d = 0; d < Q; d++) f[d] = C(0);
  } else {
    aa_read<SP>(p, A, flags, x, y, z, i, f);
  }
  export_node<C>(out, g, i, f, solid, p.gacc);
}

template <class SP>
__global__ void aa_reduce_kernel(const ReadParams p, const typename SP::S* __restrict__ A,
                                 const uint8_t* __restrict__ flags, double* out) {
  using C = typename SP::C;
  const Grid& g = p.g;
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  const int y = blockIdx.y * blockDim.y + threadIdx.y;
  const int z = blockIdx.z;
  double acc[6] = {0, 0, 0, 0, 0, 0};
  bool has = false;
  if (x < g.nx && y < g.ny) {
    const long long i = node_index(g, x, y, z);
    if (!(flags[i] & p.solid_bit)) {
      C f[Q];
      aa_read<SP>(p, A, flags, x, y, z, i, f);
      double m = 0.0;
      bool bad = false;
#pragma unroll
      for (int d = 0; d < Q; d++) {
        m += (double)f[d];
        bad = bad || !isfinite((double)f[d]);
      }
      acc[0] = m;
      acc[1] = bad ? 1.0 : 0.0;
      has = true;
    }
  }
  block_force_reduce(acc, has, out);
}

// ---- initial state ------------------------------------------------------------------------
template <class SP>
__global__ void aa_init_kernel(const InitParams p, typename SP::S* __restrict__ A,
                               const uint8_t* __restrict__ flags) {
  using C = typename SP::C;
  const Grid& g = p.g;
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  const int y = blockIdx.y * blockDim.y + threadIdx.y;
  const int z = blockIdx.z;
  if (x >= g.nx || y >= g.ny) return;
  const long long i = node_index(g, x, y, z);
  const C rho0 = C(p.rho0);
  const bool solid = (flags[i] & F_SOLID) != 0;
  if (p.f_in) {
#pragma unroll
    for (int d = 0; d < Q; d++) SP::st(A + (long long)d * g.plane + i, C(import_value(p, g, i, d)), d, rho0);
    return;
  }
  const C r = p.rho ? C(p.rho[i]) : rho0;
  const C u = p.u ? C(p.u[i]) : C(p.uni[0]);
  const C v = p.v ? C(p.v[i]) : C(p.uni[1]);
  const C w = p.w ? C(p.w[i]) : C(p.uni[2]);
#pragma unroll
  for (int d = 0; d < Q; d++)
    SP::st(A + (long long)d * g.plane + i, solid ? C(0) : feq<C>(d, r, u, v, w), d, rho0);
}

// ---- host launch templates (instantiated once per storage policy) -------------------
template <class SP, bool ODD, bool TRT, int FORCE, bool FACES>
static cudaError_t launch_one(const AAParams& p, void* A, const uint8_t* flags, dim3 grid, dim3 block,
                              cudaStream_t s) {
  if constexpr (!FACES) {
    if (p.pair) {  // 64 x 4 threads, two cells each
      const dim3 pb(64, 4, 1), pg((unsigned)(p.g.nx / 128), (unsigned)((p.g.ny + 3) / 4), (unsigned)p.g.nz);
      if constexpr (ODD && SP::DEV) {
        if (p.quad) {  // whole rows: nx / 4 threads each, 128 threads (nx at most 512) or one row
          const int rows = p.g.nx <= 512 ? 512 / p.g.nx : 1;
          const dim3 qb((unsigned)(p.g.nx / 4), (unsigned)rows, 1),
              qg(1u, (unsigned)((p.g.ny + rows - 1) / rows), (unsigned)p.g.nz);
          aa_quad_odd_kernel<TRT, FORCE><<<qg, qb, 0, s>>>(p, (__half*)A, flags);
        } else {
          aa_pair_split_kernel<SP, TRT, FORCE><<<pg, pb, 0, s>>>(p, (typename SP::S*)A, flags);
        }
      } else if constexpr (!ODD && SP::DEV) {
        if (p.quad == 2) {  // 32 x 4 threads, eight cells each (nx a multiple of 256)
          const dim3 ob(32, 4, 1), og((unsigned)(p.g.nx / 256), (unsigned)((p.g.ny + 3) / 4), (unsigned)p.g.nz);
          aa_octo_even_kernel<TRT, FORCE><<<og, ob, 0, s>>>(p, (__half*)A, flags);
        } else if (p.quad) {  // 32 x 8 threads, four cells each
          const dim3 qb(32, 8, 1), qg((unsigned)(p.g.nx / 128), (unsigned)((p.g.ny + 7) / 8), (unsigned)p.g.nz);
          aa_quad_even_kernel<TRT, FORCE><<<qg, qb, 0, s>>>(p, (__half*)A, flags);
        } else {
          aa_pair_kernel<SP, ODD, TRT, FORCE><<<pg, pb, 0, s>>>(p, (typename SP::S*)A, flags);
        }
      } else if constexpr (ODD && sizeof(typename SP::S) == 4) {
        if (p.xshuffle)
          aa_pair_odd_kernel<SP, TRT, FORCE><<<pg, pb, 0, s>>>(p, (typename SP::S*)A, flags);
        else
          aa_pair_kernel<SP, ODD, TRT, FORCE><<<pg, pb, 0, s>>>(p, (typename SP::S*)A, flags);
      } else {
        aa_pair_kernel<SP, ODD, TRT, FORCE><<<pg, pb, 0, s>>>(p, (typename SP::S*)A, flags);
      }
      return cudaGetLastError();
    }
  }
  if (p.tma.enabled) {
    auto kern = aa_tma_kernel<SP, ODD, TRT, FORCE>;
    const int smem = p.tma.stages * p.tma.stage_bytes;
    static thread_local int configured_smem = -1;  // per instantiation
    if (configured_smem != smem) {
      cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
      if (e != cudaSuccess) return e;
      configured_smem = smem;
    }
    int dev = 0, sms = 0, per_sm = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, p.tma.tw, smem);
    if (e != cudaSuccess) return e;
    if (per_sm < 1) return cudaErrorInvalidConfiguration;
    long long nb = (long long)sms * per_sm;
    if (nb > p.tma.ntiles) nb = p.tma.ntiles;
    kern<<<(unsigned)nb, p.tma.tw, smem, s>>>(p, (typename SP::S*)A, flags);
    return cudaGetLastError();
  }
  aa_step_kernel<SP, ODD, TRT, FORCE, FACES><<<grid, block, 0, s>>>(p, (typename SP::S*)A, flags);
  return cudaGetLastError();
}

template <class SP>
static cudaError_t launch_sp(const AAParams& p, void* A, const uint8_t* flags, bool odd, bool trt, int force,
                             bool faces, dim3 grid, dim3 block, cudaStream_t s) {
#define LBM_AA_CASE(O, T, F, X)                                  \
  if (odd == O && trt == T && force == F && faces == X)          \
    return launch_one<SP, O, T, F, X>(p, A, flags, grid, block, s);
#define LBM_AA_CASES(X)                 \
  LBM_AA_CASE(false, false, 0, X)       \
  LBM_AA_CASE(false, false, 1, X)       \
  LBM_AA_CASE(false, true, 0, X)        \
  LBM_AA_CASE(false, true, 1, X)        \
  LBM_AA_CASE(true, false, 0, X)        \
  LBM_AA_CASE(true, false, 1, X)        \
  LBM_AA_CASE(true, true, 0, X)         \
  LBM_AA_CASE(true, true, 1, X)
  LBM_AA_CASES(false)
  LBM_AA_CASES(true)
  // x-only acceleration (force 2): FP16-deviation storage, boxes without non-periodic
  // faces (measured on B200: +4.3 % for FP16-deviation, no gain for FP32)
  if constexpr (SP::DEV) {
    LBM_AA_CASE(false, false, 2, false)
    LBM_AA_CASE(false, true, 2, false)
    LBM_AA_CASE(true, false, 2, false)
    LBM_AA_CASE(true, true, 2, false)
  }
  if (force == 2) return launch_sp<SP>(p, A, flags, odd, trt, 1, faces, grid, block, s);
#undef LBM_AA_CASES
#undef LBM_AA_CASE
  return cudaErrorInvalidValue;
}

// Batched step: launches `blocks` persistent blocks, or, with per_sm != nullptr,
// reports how many blocks of the kernel fit on one SM.
template <class SP, bool TRT, int FORCE, bool FACES>
static cudaError_t batch_one(const BatchParams& bp, int blocks, int* per_sm, cudaStream_t s) {
  auto even = aa_batch_kernel<SP, false, TRT, FORCE, FACES>;
  auto odd = aa_batch_kernel<SP, true, TRT, FORCE, FACES>;
  if (per_sm) {
    int a = 0, b = 0;
    cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&a, even, BATCH_ITEM, 0);
    if (e == cudaSuccess) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, odd, BATCH_ITEM, 0);
    *per_sm = a < b ? a : b;
    return e;
  }
  even<<<(unsigned)blocks, BATCH_ITEM, 0, s>>>(bp);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  odd<<<(unsigned)blocks, BATCH_ITEM, 0, s>>>(bp);
  return cudaGetLastError();
}

template <class SP>
static cudaError_t batch_sp(const BatchParams& bp, bool trt, bool force, bool faces, int blocks, int* per_sm,
                            cudaStream_t s) {
#define LBM_BATCH_CASE(T, F, X) \
  if (trt == T && force == F && faces == X) return batch_one<SP, T, F, X>(bp, blocks, per_sm, s);
  LBM_BATCH_CASE(false, false, false)
  LBM_BATCH_CASE(false, false, true)
  LBM_BATCH_CASE(false, true, false)
  LBM_BATCH_CASE(false, true, true)
  LBM_BATCH_CASE(true, false, false)
  LBM_BATCH_CASE(true, false, true)
  LBM_BATCH_CASE(true, true, false)
  LBM_BATCH_CASE(true, true, true)
#undef LBM_BATCH_CASE
  return cudaErrorInvalidValue;
}

// Per-storage entry points (declared in lbm_kernels.h, dispatched in kernels_aa.cu).
#define LBM_AA_DEFINE_OPS(SP, NAME)                                                                              \
  cudaError_t aa_step_##NAME(const AAParams& p, void* A, const uint8_t* flags, bool odd, bool trt, int force,    \
                             bool faces, dim3 grid, dim3 block, cudaStream_t s) {                                \
    return launch_sp<SP>(p, A, flags, odd, trt, force, faces, grid, block, s);                                  \
  }                                                                                                              \
  cudaError_t aa_batch_##NAME(const BatchParams& bp, bool trt, bool force, bool faces, int blocks, int* per_sm, \
                              cudaStream_t s) {                                                                  \
    return batch_sp<SP>(bp, trt, force, faces, blocks, per_sm, s);                                              \
  }                                                                                                              \
  cudaError_t aa_export_##NAME(const ReadParams& p, const void* A, const uint8_t* flags, const ExportOut& out,   \
                               dim3 grid, dim3 block, cudaStream_t s) {                                          \
    aa_export_kernel<SP><<<grid, block, 0, s>>>(p, (const typename SP::S*)A, flags, out);                        \
    return cudaGetLastError();                                                                                   \
  }                                                                                                              \
  cudaError_t aa_reduce_##NAME(const ReadParams& p, const void* A, const uint8_t* flags, double* out, dim3 grid, \
                               dim3 block, cudaStream_t s) {                                                     \
    aa_reduce_kernel<SP><<<grid, block, 0, s>>>(p, (const typename SP::S*)A, flags, out);                        \
    return cudaGetLastError();                                                                                   \
  }                                                                                                              \
  cudaError_t aa_init_##NAME(const InitParams& p, void* A, const uint8_t* flags, dim3 grid, dim3 block,          \
                             cudaStream_t s) {                                                                   \
    aa_init_kernel<SP><<<grid, block, 0, s>>>(p, (typename SP::S*)A, flags);                                     \
    return cudaGetLastError();                                                                                   \
  }

}  // namespace lbm
