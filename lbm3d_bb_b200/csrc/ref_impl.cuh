// ref_impl.cuh — body of the reference-mode step kernels, included once per lattice by
// kernels_ref.cu inside a namespace that supplies Q, cx, cy, cz, opp and wgt (D3Q19 or
// D3Q27, gen_lattice_sets, Utilities.jl:945-993).  Compiled with --fmad=false.

template <class T>
struct RefT;
template <>
struct RefT<float> {
  static __device__ __forceinline__ float W(int d) { return wgt<float>(d); }
};
template <>
struct RefT<double> {
  static __device__ __forceinline__ double W(int d) { return wgt<double>(d); }
};

// compute_macros!_gpu (ComputeMacro.jl:20-40): sequential sums from zero.
template <class T>
__device__ __forceinline__ void ref_moments(const T* S, T& rho, T& u, T& v, T& w) {
  T r = T(0), mx = T(0), my = T(0), mz = T(0);
#pragma unroll
  for (int d = 0; d < Q; d++) {
    const T f = S[d];
    r += f;
    mx += f * T(cx(d));
    my += f * T(cy(d));
    mz += f * T(cz(d));
  }
  rho = r;
  u = mx / r;
  v = my / r;
  w = mz / r;
}

// BGK_collision!_gpu (Collision.jl:229-238) and TRT_collision!_gpu
// (Collision.jl:136-170), statement for statement.
template <class T, bool TRT>
__device__ __forceinline__ void ref_collide(const T* S, T* F, T rho, T ux, T uy, T uz, T om_p, T om_m) {
  if (!TRT) {
#pragma unroll
    for (int d = 0; d < Q; d++) {
      const T cu = T(cx(d)) * ux + T(cy(d)) * uy + T(cz(d)) * uz;
      const T cu2 = cu * cu;
      const T u2 = ux * ux + uy * uy + uz * uz;
      const T fe = RefT<T>::W(d) * rho * (T(1) + cu * T(3) + T(0.5) * cu2 * T(9) - T(0.5) * u2 * T(3));
      F[d] = S[d] - om_p * (S[d] - fe);
    }
  } else {
    const T u2 = ux * ux + uy * uy + uz * uz;
#pragma unroll
    for (int d = 0; d < Q; d++) {
      const T fi = S[d], fo = S[opp(d)];
      const T cu = T(cx(d)) * ux + T(cy(d)) * uy + T(cz(d)) * uz;
      const T cu2 = cu * cu;
      const T fp_eq = RefT<T>::W(d) * rho * (T(1) + T(0.5) * cu2 * T(9) - T(0.5) * u2 * T(3));
      const T fm_eq = RefT<T>::W(d) * rho * (cu * T(3));
      const T fp = T(0.5) * (fi + fo);
      const T fm = T(0.5) * (fi - fo);
      const T fpn = fp - om_p * (fp - fp_eq);
      const T fmn = fm - om_m * (fm - fm_eq);
      F[d] = fpn + fmn;
    }
  }
}

// SBB!_gpu (SolidBC.jl:181-208) for link (x, dir): value of S[opp(dir)].
template <class T>
__device__ __forceinline__ T ref_sbb(const RefParams& p, T fdir, T rho_w, int x, int y, int dir);

template <>
__device__ __forceinline__ float ref_sbb<float>(const RefParams& p, float fdir, float rho_w, int x, int y,
                                                int dir) {
  const float h = p.h;
  const float cxf = (float)cx(dir), cyf = (float)cy(dir);
  const float xlat = (((float)(x + 1) - 0.5f) * h) / h;  // x_lli ./ h (MainCore.jl:199-200)
  const float ylat = (((float)(y + 1) - 0.5f) * h) / h;
  const float xw = xlat - 0.5f * cxf, yw = ylat - 0.5f * cyf;
  const float rx = xw - (float)p.kin.center[0], ry = yw - (float)p.kin.center[1];
  const float uwx = (float)p.kin.vel[0] - (float)p.kin.omega[2] * ry;
  const float uwy = (float)p.kin.vel[1] + (float)p.kin.omega[2] * rx;
  const float cdu = cxf * uwx + cyf * uwy;
  return fdir - 2.0f * wgt<float>(dir) * rho_w * cdu * 3.0f;
}

template <>
__device__ __forceinline__ double ref_sbb<double>(const RefParams& p, double fdir, double rho_w, int x,
                                                  int y, int dir) {
  const float h = p.h;
  const double cxd = (double)cx(dir), cyd = (double)cy(dir);
  const double xlat = (double)((((float)(x + 1) - 0.5f) * h) / h);
  const double ylat = (double)((((float)(y + 1) - 0.5f) * h) / h);
  const double xw = xlat - 0.5 * cxd, yw = ylat - 0.5 * cyd;
  const double rx = xw - (double)(float)p.kin.center[0], ry = yw - (double)(float)p.kin.center[1];
  const double uwx = (double)(float)p.kin.vel[0] - (double)(float)p.kin.omega[2] * ry;
  const double uwy = (double)(float)p.kin.vel[1] + (double)(float)p.kin.omega[2] * rx;
  const double cdu = cxd * uwx + cyd * uwy;
  return fdir - 2.0 * wgt<double>(dir) * rho_w * cdu * 3.0;
}

// Interpolated bounce-back of link (x, dir), the solid at x + c_dir: the value of S[opp(dir)].
// IBB!_gpu (SolidBC.jl:253-338) as it is meant to work: phi is taken at the two ends of the
// link, the boundary node x_b and the solid node x_b + c_dir (the shipped kernel takes
// x_b - c_dir, quirk Q3); the wall lies at x_b + q c_dir; for q <= 1/2 the second point of
// the interpolation is the fluid-side neighbour x_b - c_dir (the shipped kernel reads
// nbr_lli[dir, i_b], the solid node); q is clamped to [EPS_Q, 1 - EPS_Q] with EPS_Q = 1e-4
// (a name the shipped file uses without defining it, quirk Q4).  Without a sign change of
// phi along the link the value is the moving-wall bounce-back at the half-link point
// x_b + c_dir/2.  Geometry in FP32 as the reference; the interpolation in T.
constexpr float IBB_EPS_Q = 1e-4f;

__device__ __forceinline__ float ibb_phi(const IbbGeom& b, float x, float y) {
  if (b.shape == LBM_BODY_CYLINDER_Z) return phi_cylinder(x, y, b.xc, b.yc, b.R);
  return phi_airfoil(x, y, b.xc, b.yc, b.ct, b.st, b.chord, b.m, b.p, b.t, b.x_int, b.x_le);
}

template <class T>
__device__ __forceinline__ T ref_ibb(const RefParams& p, const T* __restrict__ Fp, T rho_w, int x, int y, int z,
                                     long long i, int dir) {
  const Grid& g = p.g;
  const float h = p.h;
  const float cxf = (float)cx(dir), cyf = (float)cy(dir);
  const float xb = (((float)(x + 1) - 0.5f) * h) / h;  // x_lli ./ h (MainCore.jl:199-200)
  const float yb = (((float)(y + 1) - 0.5f) * h) / h;
  const float phib = ibb_phi(p.ibb, xb, yb);
  const float phis = ibb_phi(p.ibb, xb + cxf, yb + cyf);
  const float denom = phib - phis;
  const bool no_brkt = (phib <= 0.0f) || (phis >= 0.0f) || (fabsf(denom) < 1e-8f);
  const float q = no_brkt ? 0.5f : fminf(fmaxf(phib / denom, IBB_EPS_Q), 1.0f - IBB_EPS_Q);
  // moving-wall term at the wall point x_w = x_b + q c_dir (uw_at_wall_lat_planar)
  const float xw = xb + q * cxf, yw = yb + q * cyf;
  const float rx = xw - (float)p.kin.center[0], ry = yw - (float)p.kin.center[1];
  const float uwx = (float)p.kin.vel[0] - (float)p.kin.omega[2] * ry;
  const float uwy = (float)p.kin.vel[1] + (float)p.kin.omega[2] * rx;
  const float cdu = cxf * uwx + cyf * uwy;
  const T corr = T(2) * RefT<T>::W(dir) * rho_w * T(cdu) * T(3);
  const T fdir = Fp[(long long)dir * g.plane + i];
  if (no_brkt) return fdir - corr;
  const T tq = T(q);
  if (q <= 0.5f) {
    // fluid-side neighbour x_b - c_dir, across the periodic z axis as in streaming (the
    // shipped nbr_lli stops at the z ends, which would send every link with c_z != 0 in the
    // end planes of an extruded box to the same-node branch, unstable for small q);
    // outside the x/y range the same-node branch
    const int fx = x - cx(dir), fy = y - cy(dir), fz = (z - cz(dir) + g.nz) % g.nz;
    if (fx >= 0 && fx < g.nx && fy >= 0 && fy < g.ny) {
      const T ff = Fp[(long long)dir * g.plane + node_index(g, fx, fy, fz)];
      return T(2) * tq * fdir + (T(1) - T(2) * tq) * ff - corr;
    }
  }
  const T fopp = Fp[(long long)opp(dir) * g.plane + i];
  return (T(0.5) / tq) * fdir + ((T(2) * tq - T(1)) / (T(2) * tq)) * fopp - corr;
}

// Pull S_n at node (x,y,z) from F_{n-1} and apply the solid and face conditions
// (Streaming.jl:82-111, OtherBC.jl:65-82, SolidBC.jl:160-210, OtherBC.jl:112-169),
// accumulating the momentum exchange (MEA.jl:93-113).
template <class T>
__device__ __forceinline__ void ref_pull(const RefParams& p, const T* __restrict__ Fp,
                                         const T* __restrict__ Rp, const uint8_t* __restrict__ flags,
                                         int x, int y, int z, long long i, T* S, double* acc, bool& has) {
  const Grid& g = p.g;
  const long long nxl = g.nx, nxy = (long long)g.nx * g.ny;
  const int zm = z == 0 ? g.nz - 1 : z - 1, zp = z == g.nz - 1 ? 0 : z + 1;
#pragma unroll
  for (int d = 0; d < Q; d++) {
    const int sx = x - cx(d), sy = y - cy(d);
    const int sz = cz(d) == 1 ? zm : (cz(d) == -1 ? zp : z);
    long long src = i;  // x/y out of domain: same node, same direction (Utilities.jl:773-776)
    if (sx >= 0 && sx < g.nx && sy >= 0 && sy < g.ny) src = sx + nxl * sy + nxy * sz;
    S[d] = Fp[(long long)d * g.plane + src];
  }
  const uint8_t fl = flags[i];
  const bool solid = (fl & p.solid_bit) != 0;
  const bool on_face = (x == 0) || (x == g.nx - 1) || (y == 0) || (y == g.ny - 1);
  const bool near = !solid && (fl & F_NEAR);
  if (!(near || on_face)) return;
  const T rp = Rp[i];
  uint32_t links = 0;
  if (near) {
#pragma unroll
    for (int dir = 0; dir < Q; dir++) {
      const int nx_ = x + cx(dir), ny_ = y + cy(dir), nz_ = z + cz(dir);
      // nbr_lli: -1 outside the global domain, z included (Utilities.jl:559-569)
      if (nx_ < 0 || nx_ >= g.nx || ny_ < 0 || ny_ >= g.ny || nz_ < 0 || nz_ >= g.nz) continue;
      if (!(flags[nx_ + nxl * ny_ + nxy * nz_] & p.solid_bit)) continue;
      links |= 1u << dir;
      if (p.solid_bc == LBM_SOLID_IBB) {
        S[opp(dir)] = ref_ibb<T>(p, Fp, rp, x, y, z, i, dir);
      } else {
        const T fdir = Fp[(long long)dir * g.plane + i];
        S[opp(dir)] = ref_sbb<T>(p, fdir, rp, x, y, dir);
      }
    }
  }
  if (on_face) {
    const T up = Rp[g.N + i], vp = Rp[2 * g.N + i], wp = Rp[3 * g.N + i];
    const T U = T(p.U), V = T(p.V), W = T(p.W);
    // velocity list: inlet x=1 (c_x>0), y=1 (c_y>0), y=Ny (c_y<0) — OtherBC.jl:139-148
#pragma unroll
    for (int dir = 0; dir < Q; dir++) {
      const bool vel = (x == 0 && cx(dir) > 0) || (y == 0 && cy(dir) > 0) || (y == g.ny - 1 && cy(dir) < 0);
      if (vel) {
        const T cu = T(cx(dir)) * (-U) + T(cy(dir)) * (-V) + T(cz(dir)) * (-W);
        S[dir] = Fp[(long long)opp(dir) * g.plane + i] - T(2) * RefT<T>::W(dir) * rp * cu * T(3);
      }
    }
    // pressure list: outlet x=Nx (c_x<0) — OtherBC.jl:153-165; written last, so it
    // wins where both lists name a slot
    if (x == g.nx - 1) {
#pragma unroll
      for (int dir = 0; dir < Q; dir++) {
        if (cx(dir) < 0) {
          const T cu = T(cx(dir)) * up + T(cy(dir)) * vp + T(cz(dir)) * wp;
          const T cu2 = cu * cu;
          const T uu2 = up * up + vp * vp + wp * wp;
          S[dir] = -Fp[(long long)opp(dir) * g.plane + i] +
                   T(2) * RefT<T>::W(dir) * rp * (T(1) + T(0.5) * cu2 * T(9) - T(0.5) * uu2 * T(3));
        }
      }
    }
  }
  if (links && p.compute_force) {
    const double hl = (double)p.h;
    const double rx = (double)((((float)(x + 1) - 0.5f) * p.h) / p.h) - (double)(float)p.kin.center[0];
    const double ry = (double)((((float)(y + 1) - 0.5f) * p.h) / p.h) - (double)(float)p.kin.center[1];
    const double rz = (z + 0.5) - p.kin.center[2];
    (void)hl;
#pragma unroll
    for (int dir = 0; dir < Q; dir++) {
      if (!((links >> dir) & 1u)) continue;
      const double t = (double)Fp[(long long)dir * g.plane + i] + (double)S[opp(dir)];
      const double fx = t * cx(dir), fy = t * cy(dir), fz = t * cz(dir);
      acc[0] += fx;
      acc[1] += fy;
      acc[2] += fz;
      acc[3] += ry * fz - rz * fy;
      acc[4] += rz * fx - rx * fz;
      acc[5] += rx * fy - ry * fx;
    }
    has = true;
  }
}

template <class T, bool TRT>
__global__ void __launch_bounds__(256) ref_step_kernel(const __grid_constant__ RefParams p,
                                                       const T* __restrict__ Fp, const T* __restrict__ Rp,
                                                       T* __restrict__ Fn, T* __restrict__ Rn,
                                                       const uint8_t* __restrict__ flags) {
  const Grid& g = p.g;
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  const int y = blockIdx.y * blockDim.y + threadIdx.y;
  const int z = blockIdx.z;
  double acc[6] = {0, 0, 0, 0, 0, 0};
  bool has = false;
  clear_record(p.zero_next);  // the next step's force record (read by the next launch only)
  if (x < g.nx && y < g.ny) {
    const long long i = node_index(g, x, y, z);
    T S[Q];
    ref_pull<T>(p, Fp, Rp, flags, x, y, z, i, S, acc, has);
    T rho, u, v, w;
    ref_moments<T>(S, rho, u, v, w);
    Rn[i] = rho;
    Rn[g.N + i] = u;
    Rn[2 * g.N + i] = v;
    Rn[3 * g.N + i] = w;
    T F[Q];
    ref_collide<T, TRT>(S, F, rho, u, v, w, T(p.omega_p), T(p.omega_m));
#pragma unroll
    for (int d = 0; d < Q; d++) Fn[(long long)d * g.plane + i] = F[d];
  }
  if (p.compute_force) block_force_reduce(acc, has, p.force + block_stripe());
}

// Populations (SoA or the reference's f[d + q*node]) and moments of one node for export.
template <class T>
__device__ __forceinline__ void ref_export_node(const ExportOut& o, const Grid& g, long long i, const T* f) {
  if (o.f) {
#pragma unroll
    for (int d = 0; d < Q; d++) {
      const long long k = o.f_layout == LBM_LAYOUT_SOA ? (long long)d * g.N + i : (long long)d + (long long)Q * i;
      put<T>(o.f, k, o.f_dtype, f[d]);
    }
  }
  if (o.rho || o.u || o.v || o.w) {
    T r = f[0], jx = T(0), jy = T(0), jz = T(0);
#pragma unroll
    for (int d = 1; d < Q; d++) r += f[d];
#pragma unroll
    for (int d = 0; d < Q; d++) {
      jx += f[d] * T(cx(d));
      jy += f[d] * T(cy(d));
      jz += f[d] * T(cz(d));
    }
    if (o.rho) put<T>(o.rho, i, o.m_dtype, r);
    if (o.u) put<T>(o.u, i, o.m_dtype, jx / r);
    if (o.v) put<T>(o.v, i, o.m_dtype, jy / r);
    if (o.w) put<T>(o.w, i, o.m_dtype, jz / r);
  }
}

template <class T>
__global__ void ref_export_kernel(const __grid_constant__ RefParams p, const T* __restrict__ Fp,
                                  const T* __restrict__ Rp, int direct, const uint8_t* __restrict__ flags,
                                  ExportOut out, double* mass) {
  const Grid& g = p.g;
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  const int y = blockIdx.y * blockDim.y + threadIdx.y;
  const int z = blockIdx.z;
  double acc[6] = {0, 0, 0, 0, 0, 0};
  bool has = false;
  if (x < g.nx && y < g.ny) {
    const long long i = node_index(g, x, y, z);
    T S[Q];
    if (direct) {
#pragma unroll
      for (int d = 0; d < Q; d++) S[d] = Fp[(long long)d * g.plane + i];
    } else {
      double dummy[6] = {0, 0, 0, 0, 0, 0};
      bool hd = false;
      RefParams q = p;
      q.compute_force = 0;
      ref_pull<T>(q, Fp, Rp, flags, x, y, z, i, S, dummy, hd);
    }
    if (mass) {
      double m = 0.0;
      bool bad = false;
#pragma unroll
      for (int d = 0; d < Q; d++) {
        m += (double)S[d];
        bad = bad || !isfinite((double)S[d]);
      }
      acc[0] = m;
      acc[1] = bad ? 1.0 : 0.0;
      has = true;
    } else {
      ref_export_node<T>(out, g, i, S);
    }
  }
  if (mass) block_force_reduce(acc, has, mass);
}

template <class T, bool TRT>
__global__ void ref_prepare_kernel(const __grid_constant__ RefParams p, const T* __restrict__ S0,
                                   T* __restrict__ F, T* __restrict__ R) {
  const Grid& g = p.g;
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  const int y = blockIdx.y * blockDim.y + threadIdx.y;
  const int z = blockIdx.z;
  if (x >= g.nx || y >= g.ny) return;
  const long long i = node_index(g, x, y, z);
  T S[Q];
#pragma unroll
  for (int d = 0; d < Q; d++) S[d] = S0[(long long)d * g.plane + i];
  T rho, u, v, w;
  ref_moments<T>(S, rho, u, v, w);
  R[i] = rho;
  R[g.N + i] = u;
  R[2 * g.N + i] = v;
  R[3 * g.N + i] = w;
  T Fo[Q];
  ref_collide<T, TRT>(S, Fo, rho, u, v, w, T(p.omega_p), T(p.omega_m));
#pragma unroll
  for (int d = 0; d < Q; d++) F[(long long)d * g.plane + i] = Fo[d];
}

// initialize_f_gpu (Initialization.jl:27-41) with the caller's velocity field.
template <class T>
__global__ void ref_init_kernel(const InitParams p, T* __restrict__ S) {
  const Grid& g = p.g;
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  const int y = blockIdx.y * blockDim.y + threadIdx.y;
  const int z = blockIdx.z;
  if (x >= g.nx || y >= g.ny) return;
  const long long i = node_index(g, x, y, z);
  if (p.f_in) {
#pragma unroll
    for (int d = 0; d < Q; d++) S[(long long)d * g.plane + i] = T(import_value(p, g, i, d));
    return;
  }
  const T r = p.rho ? T(p.rho[i]) : T(p.rho0);
  const T ux = p.u ? T(p.u[i]) : T(p.uni[0]);
  const T uy = p.v ? T(p.v[i]) : T(p.uni[1]);
  const T uz = p.w ? T(p.w[i]) : T(p.uni[2]);
#pragma unroll
  for (int d = 0; d < Q; d++) {
    const T cu = T(cx(d)) * ux + T(cy(d)) * uy + T(cz(d)) * uz;
    const T u2 = ux * ux + uy * uy + uz * uz;
    const T cu2 = cu * cu;
    S[(long long)d * g.plane + i] =
        RefT<T>::W(d) * r * (T(1) + cu * T(3) + T(0.5) * cu2 * T(9) - T(0.5) * u2 * T(3));
  }
}

template <class T>
__global__ void ref_macros_kernel(const Grid g, const T* __restrict__ R, ExportOut out) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  const int y = blockIdx.y * blockDim.y + threadIdx.y;
  const int z = blockIdx.z;
  if (x >= g.nx || y >= g.ny) return;
  const long long i = node_index(g, x, y, z);
  if (out.rho) put<T>(out.rho, i, out.m_dtype, R[i]);
  if (out.u) put<T>(out.u, i, out.m_dtype, R[g.N + i]);
  if (out.v) put<T>(out.v, i, out.m_dtype, R[2 * g.N + i]);
  if (out.w) put<T>(out.w, i, out.m_dtype, R[3 * g.N + i]);
}

