// lbm_oracle.cpp — CPU restatement of the LBM3D_BB single-domain time step.
//
// TEST INFRASTRUCTURE ONLY (parity checker and timed CPU baseline); parity is
// UNPINNED — see lbm_oracle.h.  Build: oracle/Makefile (-O3 -ffp-contract=off
// -fopenmp), so that FP32 expressions round exactly as written.
//
// Formulation: two arrays, "collide every node, then pull-stream with boundary
// overrides", i.e. the reference's own sequence (MainCore.jl:245-379).  It is
// deliberately not the in-place AA scheme the GPU library uses, so the two are
// independent restatements.
//
// Reference mode follows, statement by statement:
//   lattice               Utilities.jl:949-960
//   BGK collision         Collision.jl:227-239      TRT collision  Collision.jl:129-171
//   pull streaming        Utilities.jl:734-790 + Streaming.jl:82-111
//   z-periodic copy       Utilities.jl:860-898 + OtherBC.jl:65-82
//   solid flags           Geometry.jl:49-87 (cylinder :73, NACA band :75-82, helpers :321-356)
//   boundary flags        Geometry.jl:122-148 with nbr_lli of Utilities.jl:555-572 (no z wrap)
//   link CSR              Geometry.jl:181-311 (node-major, direction-minor, 1-based)
//   SBB moving wall       SolidBC.jl:160-210
//   face BCs              Utilities.jl:795-855 + OtherBC.jl:112-169
//   momentum exchange     MEA.jl:76-116 (accumulated in FP64 here)
//   macros                ComputeMacro.jl:11-48
//   init                  Initialization.jl:11-47 (velocity field supplied by caller)
// Quirks kept: solids are collided/streamed as virtual fluid (Collision.jl:227-228,
// no refill, Motion.jl:72-93); the SBB wall point is x_i - c/2 (SolidBC.jl:195-196);
// x/y out-of-domain stream sources fall back to the same node and direction
// (Utilities.jl:773-776) before the face BCs overwrite them; no bounce-back link
// crosses the z-periodic boundary (nbr_lli is -1 there, Utilities.jl:559-569);
// where a velocity entry and a pressure entry name the same slot (outlet corners,
// OtherBC.jl:138-166 race) the pressure entry wins.
//
// Config mode is the configurable physics of the same step: per-face kinds,
// periodic axes, Guo forcing, static + one moving body with equilibrium refill
// of uncovered nodes, BB links across periodic boundaries, solids not evolved.
#include "lbm_oracle.h"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

// D3Q19 of gen_lattice_sets, Utilities.jl:949-960, 0-based.
const int CX[19] = {1, -1, 0, 0, 0, 0, 1, -1, 1, -1, 0, 0, 1, -1, 1, -1, 0, 0, 0};
const int CY[19] = {0, 0, 1, -1, 0, 0, 1, -1, 0, 0, 1, -1, -1, 1, 0, 0, 1, -1, 0};
const int CZ[19] = {0, 0, 0, 0, 1, -1, 0, 0, 1, -1, 1, -1, 0, 0, -1, 1, -1, 1, 0};
const int OPP[19] = {1, 0, 3, 2, 5, 4, 7, 6, 9, 8, 11, 10, 13, 12, 15, 14, 17, 16, 18};
const int Q = 19;

template <class T>
T weight(int d) {  // Float32.(W) of the rationals 1//18, 1//36, 1//3
  return d < 6 ? T(1) / T(18) : (d < 18 ? T(1) / T(36) : T(1) / T(3));
}

// D3Q27 of gen_lattice_sets, Utilities.jl:962-976, 0-based: the D3Q19 directions first,
// then the eight corners, rest last; opposite pairs (2k, 2k+1).
const int CX27[27] = {1, -1, 0, 0, 0, 0, 1, -1, 1, -1, 0, 0, 1, -1, 1, -1, 0, 0, 1, -1, 1, -1, 1, -1, -1, 1, 0};
const int CY27[27] = {0, 0, 1, -1, 0, 0, 1, -1, 0, 0, 1, -1, -1, 1, 0, 0, 1, -1, 1, -1, 1, -1, -1, 1, 1, -1, 0};
const int CZ27[27] = {0, 0, 0, 0, 1, -1, 0, 0, 1, -1, 1, -1, 0, 0, -1, 1, -1, 1, 1, -1, -1, 1, 1, -1, 1, -1, 0};

template <class T>
T weight27(int d) {  // Float32.(W) of 2//27, 1//54, 1//216, 8//27
  return d < 6 ? T(2) / T(27) : (d < 18 ? T(1) / T(54) : (d < 26 ? T(1) / T(216) : T(8) / T(27)));
}

struct Body {
  lbm_body b;
};

// ---- geometry predicates -------------------------------------------------------
// FP32 with the reference's operation order (Geometry.jl:66-83); compiled with
// -ffp-contract=off so no multiply-add is fused.
bool inside_cylinder_f32(float x, float y, float xc, float yc, float R) {
  float dx = x - xc;
  float dy = y - yc;
  float R2 = R * R;  // SolidMaskState.R2 = R*R (Geometry.jl:30)
  return (dx * dx + dy * dy) <= (R2 + 1e-6f * R2);
}

// NACA 4-digit helpers (Geometry.jl:321-356).  cos(atan(s)) is evaluated as
// 1/sqrt(1+s*s) (equal in exact arithmetic) so that CPU and GPU round alike;
// x^4 is (x*x)*(x*x).
void naca_upper_lower_f32(float x, float c, float m, float p, float t, float x_int, float* yL,
                          float* yU) {
  float xbar = x / c;
  float xbi = std::max(0.0f, x_int * xbar);
  float rt = std::sqrt(xbi);
  float x2 = xbi * xbi;
  float x3 = x2 * xbi;
  float x4 = x2 * x2;
  float yt = 5.0f * t * c *
             (0.2969f * rt - 0.1260f * xbi - 0.3516f * x2 + 0.2843f * x3 - 0.1015f * x4);
  float yc = 0.0f, dycb = 0.0f;
  if (m == 0.0f || p == 0.0f) {
    yc = 0.0f;
    dycb = 0.0f;
  } else if (xbar < p) {
    yc = m / (p * p) * (2.0f * p * xbar - xbar * xbar);
    dycb = 2.0f * m / (p * p) * (p - xbar);
  } else {
    float den = 1.0f - p;
    float den2 = den * den;
    yc = m / den2 * ((1.0f - 2.0f * p) + 2.0f * p * xbar - xbar * xbar);
    dycb = 2.0f * m / den2 * (p - xbar);
  }
  float s = dycb / c;
  float cz = 1.0f / std::sqrt(1.0f + s * s);
  *yU = yc + yt * cz;
  *yL = yc - yt * cz;
}

bool inside_naca_f32(float x, float y, float xc, float yc, float ct, float st, const lbm_body& b) {
  float dx = x - xc, dy = y - yc;
  float xB = ct * dx + st * dy;   // _rot_to_body (Geometry.jl:321-323)
  float yB = -st * dx + ct * dy;
  float chord = (float)b.chord;
  float xle = xB + (float)b.x_le_offset;
  if (!(0.0f <= xle && xle <= chord)) return false;
  float yL, yU;
  naca_upper_lower_f32(xle, chord, (float)b.naca_m, (float)b.naca_p, (float)b.naca_t,
                       (float)b.x_int, &yL, &yU);
  float tol = 1e-6f * chord;
  return (yL - tol <= yB) && (yB <= yU + tol);
}

// phi_cylinder_lat (Geometry.jl:365-369) and phi_airfoil_lat (Geometry.jl:372-392), FP32;
// hypot(a, b) is evaluated as sqrt(a*a + b*b).
float phi_cylinder_f32(float x, float y, float xc, float yc, float R) {
  float dx = x - xc, dy = y - yc;
  return std::sqrt(dx * dx + dy * dy) - R;
}

float phi_airfoil_f32(float xw, float yw, float xc, float yc, float ct, float st, float chord, float m,
                      float p, float t, float x_int, float x_le_offset) {
  float dx = xw - xc, dy = yw - yc;
  float xB = ct * dx + st * dy;
  float yB = -st * dx + ct * dy;
  float xle = xB + x_le_offset;
  if (xle < 0.0f) return std::sqrt(xle * xle + yB * yB);  // ahead of the leading edge
  if (xle > chord) {                                      // behind the trailing edge
    float a = xle - chord;
    return std::sqrt(a * a + yB * yB);
  }
  float yL, yU;
  naca_upper_lower_f32(xle, chord, m, p, t, x_int, &yL, &yU);
  if ((yB >= yL) && (yB <= yU)) return -std::min(yU - yB, yB - yL);
  return (yB > yU) ? (yB - yU) : (yL - yB);
}

double min_image(double d, int n, bool periodic) {
  if (!periodic) return d;
  double hn = 0.5 * n;
  if (d > hn) d -= n;
  else if (d < -hn) d += n;
  return d;
}

bool inside_sphere(double dx, double dy, double dz, double r) {
  return (dx * dx + dy * dy) + dz * dz <= r * r;
}

bool inside_ellipsoid(double dx, double dy, double dz, const double* rot, const double* semi) {
  // body = rot^T * world (rot row-major body->world)
  double b0 = (rot[0] * dx + rot[3] * dy) + rot[6] * dz;
  double b1 = (rot[1] * dx + rot[4] * dy) + rot[7] * dz;
  double b2 = (rot[2] * dx + rot[5] * dy) + rot[8] * dz;
  double q0 = b0 / semi[0], q1 = b1 / semi[1], q2 = b2 / semi[2];
  return (q0 * q0 + q1 * q1) + q2 * q2 <= 1.0;
}

template <class T>
struct Sim {
  lbm_config cfg;
  int nx, ny, nz;
  int64_t N;
  bool per[3];
  std::string err;
  std::vector<T> S, P;             // S: pre-collision state; P: post-collision
  std::vector<T> rho, ux, uy, uz;  // reference mode: stored macros of S
  std::vector<uint8_t> solid, solid_prev, moving, static_solid;
  std::vector<Body> bodies;
  int moving_idx = -1;
  bool any_body = false;
  double torque_center[3] = {0, 0, 0};  // first body's centre when no body moves
  lbm_pose pose_n{}, pose_half{};
  bool have_pose = false;
  int64_t nstep = 0;
  std::vector<double> force_hist;  // 6 per step
  // the lattice of this run (these members shadow the D3Q19 tables at namespace scope)
  int Q = 19;
  int CX[27], CY[27], CZ[27], OPP[27];
  T w[27];

  bool ref() const { return cfg.mode == LBM_MODE_REFERENCE; }

  int init(const lbm_config* c) {
    cfg = *c;
    nx = c->nx;
    ny = c->ny;
    nz = c->nz;
    if (c->q != 19 && !(c->q == 27 && c->mode == LBM_MODE_REFERENCE)) {
      err = "q=19, or q=27 in reference mode";
      return LBM_ERR_UNSUPPORTED;
    }
    Q = c->q;
    for (int d = 0; d < Q; d++) {
      CX[d] = Q == 19 ? ::CX[d] : CX27[d];
      CY[d] = Q == 19 ? ::CY[d] : CY27[d];
      CZ[d] = Q == 19 ? ::CZ[d] : CZ27[d];
      OPP[d] = d == Q - 1 ? d : (d ^ 1);
    }
    if (nx < 2 || ny < 2 || nz < 1) {
      err = "bad dimensions";
      return LBM_ERR_ARG;
    }
    N = (int64_t)nx * ny * nz;
    if (ref()) {
      per[0] = per[1] = false;
      per[2] = true;
      if (cfg.h == 0.0) cfg.h = 1.0;
    } else {
      for (int a = 0; a < 3; a++) per[a] = (c->face[2 * a] == LBM_FACE_PERIODIC);
      if (cfg.h == 0.0) cfg.h = 1.0;
    }
    for (int d = 0; d < Q; d++) w[d] = Q == 19 ? weight<T>(d) : weight27<T>(d);
    S.assign((size_t)Q * N, T(0));
    P.assign((size_t)Q * N, T(0));
    if (ref()) {
      rho.assign(N, T(0));
      ux.assign(N, T(0));
      uy.assign(N, T(0));
      uz.assign(N, T(0));
    }
    solid.assign(N, 0);
    solid_prev.assign(N, 0);
    moving.assign(N, 0);
    static_solid.assign(N, 0);
    return LBM_OK;
  }

  int64_t idx(int x, int y, int z) const { return x + (int64_t)nx * (y + (int64_t)ny * z); }

  // ---- rasterisation -------------------------------------------------------------
  // Whether node (x,y,z) lies inside body b at pose (c, ct, st, rot).
  bool inside(const lbm_body& b, int x, int y, int z, const double* c, double ct, double st,
              const double* rot) const {
    switch (b.kind) {
      case LBM_BODY_CYLINDER_Z: {
        float h = (float)cfg.h;
        float xl = ((float)(x + 1) - 0.5f) * h;  // Utilities.jl:550 (1-based ix)
        float yl = ((float)(y + 1) - 0.5f) * h;
        return inside_cylinder_f32(xl, yl, (float)c[0], (float)c[1], (float)b.radius);
      }
      case LBM_BODY_NACA_Z: {
        float h = (float)cfg.h;
        float xl = ((float)(x + 1) - 0.5f) * h;
        float yl = ((float)(y + 1) - 0.5f) * h;
        return inside_naca_f32(xl, yl, (float)c[0], (float)c[1], (float)ct, (float)st, b);
      }
      case LBM_BODY_SPHERE: {
        double dx = min_image((x + 0.5) - c[0], nx, per[0]);
        double dy = min_image((y + 0.5) - c[1], ny, per[1]);
        double dz = min_image((z + 0.5) - c[2], nz, per[2]);
        return inside_sphere(dx, dy, dz, b.radius);
      }
      case LBM_BODY_ELLIPSOID: {
        double dx = min_image((x + 0.5) - c[0], nx, per[0]);
        double dy = min_image((y + 0.5) - c[1], ny, per[1]);
        double dz = min_image((z + 0.5) - c[2], nz, per[2]);
        return inside_ellipsoid(dx, dy, dz, rot, b.semi);
      }
    }
    return false;
  }

  void raster(const lbm_body& b, const double* c, double ct, double st, const double* rot,
              std::vector<uint8_t>& out) {
    // 3-D shapes: only the box of radius max(radius, semi-axes) + 1 around the centre can
    // hold inside nodes (whole axis when the box reaches around a periodic axis)
    int lo[3] = {0, 0, 0}, hi[3] = {nx - 1, ny - 1, nz - 1};
    const bool box = b.kind == LBM_BODY_SPHERE || b.kind == LBM_BODY_ELLIPSOID;
    if (box) {
      double r = b.kind == LBM_BODY_SPHERE ? b.radius : std::max(b.semi[0], std::max(b.semi[1], b.semi[2]));
      const int n3[3] = {nx, ny, nz};
      for (int a = 0; a < 3; a++) {
        int l = (int)std::floor(c[a] - r - 1.0), h = (int)std::ceil(c[a] + r + 1.0);
        if (!per[a]) {
          l = std::max(l, 0);
          h = std::min(h, n3[a] - 1);
        } else if (h - l + 1 >= n3[a]) {
          l = 0;
          h = n3[a] - 1;
        }
        lo[a] = l;
        hi[a] = h;
      }
    }
#pragma omp parallel for schedule(static)
    for (int zz = lo[2]; zz <= hi[2]; zz++)
      for (int yy = lo[1]; yy <= hi[1]; yy++)
        for (int xx = lo[0]; xx <= hi[0]; xx++) {
          const int x = ((xx % nx) + nx) % nx, y = ((yy % ny) + ny) % ny, z = ((zz % nz) + nz) % nz;
          if (inside(b, x, y, z, c, ct, st, rot)) out[idx(x, y, z)] = 1;
        }
  }

  // Bounding box of the solid nodes, grown by one node (the links and the bounce-back
  // flags lie inside it); a whole axis when the grown box reaches around a periodic axis.
  // Returns false when there is no solid node.
  bool link_box(int lo[3], int hi[3]) const {
    int l0 = nx, l1 = ny, l2 = nz, h0 = -1, h1 = -1, h2 = -1;
#pragma omp parallel for schedule(static) reduction(min : l0, l1, l2) reduction(max : h0, h1, h2)
    for (int z = 0; z < nz; z++)
      for (int y = 0; y < ny; y++)
        for (int x = 0; x < nx; x++)
          if (solid[idx(x, y, z)]) {
            l0 = std::min(l0, x), h0 = std::max(h0, x);
            l1 = std::min(l1, y), h1 = std::max(h1, y);
            l2 = std::min(l2, z), h2 = std::max(h2, z);
          }
    if (h0 < 0) return false;
    const int n3[3] = {nx, ny, nz}, L[3] = {l0, l1, l2}, H[3] = {h0, h1, h2};
    for (int a = 0; a < 3; a++) {
      lo[a] = L[a] - 1;
      hi[a] = H[a] + 1;
      if (lo[a] < 0 || hi[a] >= n3[a]) {
        // a link may cross a periodic boundary (config mode; reference mode wraps z only
        // in streaming, never in the link set, so clamping is exact there)
        if (per[a] && !ref()) {
          lo[a] = 0;
          hi[a] = n3[a] - 1;
        } else {
          lo[a] = std::max(lo[a], 0);
          hi[a] = std::min(hi[a], n3[a] - 1);
        }
      }
    }
    return true;
  }

  static void body_rot(const lbm_body& b, double* rot, double* ct, double* st) {
    bool zero = true;
    for (int i = 0; i < 9; i++) zero = zero && (b.rot[i] == 0.0);
    if (zero) {
      for (int i = 0; i < 9; i++) rot[i] = (i % 4 == 0) ? 1.0 : 0.0;
    } else {
      for (int i = 0; i < 9; i++) rot[i] = b.rot[i];
    }
    *ct = rot[0];
    *st = rot[3];
  }

  // centre the momentum-exchange torque refers to
  void lever_center(double* c) const {
    for (int a = 0; a < 3; a++) c[a] = moving_idx >= 0 ? pose_half.center[a] : torque_center[a];
  }

  int add_body(const lbm_body* b) {
    if (!any_body) {
      for (int a = 0; a < 3; a++) torque_center[a] = b->center[a];
      any_body = true;
    }
    if (b->moving) {
      if (moving_idx >= 0) {
        err = "at most one moving body";
        return LBM_ERR_ARG;
      }
      bodies.push_back(Body{*b});
      moving_idx = (int)bodies.size() - 1;
      for (int a = 0; a < 3; a++) pose_half.center[a] = b->center[a];
      // initial rasterisation at the body's own pose (replaced by update_body)
      double rot[9], ct, st;
      body_rot(*b, rot, &ct, &st);
      std::fill(moving.begin(), moving.end(), 0);
      raster(*b, b->center, ct, st, rot, moving);
    } else {
      bodies.push_back(Body{*b});
      double rot[9], ct, st;
      body_rot(*b, rot, &ct, &st);
      raster(*b, b->center, ct, st, rot, static_solid);
    }
    for (int64_t i = 0; i < N; i++) {
      solid[i] = static_solid[i] | moving[i];
      solid_prev[i] = solid[i];
    }
    return LBM_OK;
  }

  int add_spheres(int count, const double* xyzr) {
    if (ref()) {
      err = "lbm_add_spheres is config-mode only";
      return LBM_ERR_ARG;
    }
    if (!any_body && count > 0) {
      for (int a = 0; a < 3; a++) torque_center[a] = xyzr[a];
      any_body = true;
    }
    for (int s = 0; s < count; s++) {
      double c[3] = {xyzr[4 * s], xyzr[4 * s + 1], xyzr[4 * s + 2]};
      double r = xyzr[4 * s + 3];
      // bounding box (with periodic wrap)
      int lo[3], hi[3];
      int n3[3] = {nx, ny, nz};
      for (int a = 0; a < 3; a++) {
        lo[a] = (int)std::floor(c[a] - r - 1.0);
        hi[a] = (int)std::ceil(c[a] + r + 1.0);
        if (!per[a]) {
          lo[a] = std::max(lo[a], 0);
          hi[a] = std::min(hi[a], n3[a] - 1);
        } else if (hi[a] - lo[a] + 1 >= n3[a]) {
          lo[a] = 0;
          hi[a] = n3[a] - 1;
        }
      }
      for (int zz = lo[2]; zz <= hi[2]; zz++)
        for (int yy = lo[1]; yy <= hi[1]; yy++)
          for (int xx = lo[0]; xx <= hi[0]; xx++) {
            int x = ((xx % nx) + nx) % nx, y = ((yy % ny) + ny) % ny, z = ((zz % nz) + nz) % nz;
            double dx = min_image((x + 0.5) - c[0], nx, per[0]);
            double dy = min_image((y + 0.5) - c[1], ny, per[1]);
            double dz = min_image((z + 0.5) - c[2], nz, per[2]);
            if (inside_sphere(dx, dy, dz, r)) static_solid[idx(x, y, z)] = 1;
          }
    }
    for (int64_t i = 0; i < N; i++) {
      solid[i] = static_solid[i] | moving[i];
      solid_prev[i] = solid[i];
    }
    return LBM_OK;
  }

  int update_body(const lbm_pose* pn, const lbm_pose* ph) {
    pose_n = *pn;
    pose_half = ph ? *ph : *pn;
    have_pose = true;
    if (moving_idx < 0) return LBM_OK;
    const lbm_body& b = bodies[moving_idx].b;
    std::fill(moving.begin(), moving.end(), 0);
    double rot[9];
    bool zero = true;
    for (int i = 0; i < 9; i++) zero = zero && (pn->rot[i] == 0.0);
    for (int i = 0; i < 9; i++) rot[i] = zero ? ((i % 4 == 0) ? 1.0 : 0.0) : pn->rot[i];
    raster(b, pn->center, pn->cos_theta, pn->sin_theta, rot, moving);
    // solid_prev keeps the flags the last completed step used (set at its end)
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < N; i++) solid[i] = static_solid[i] | moving[i];
    return LBM_OK;
  }

  // neighbour of node (x,y,z) in direction c (+1: x + c_d, -1: x - c_d).  Returns
  // -1 when outside a non-periodic axis (or any axis but z in reference mode).
  int64_t neighbour(int x, int y, int z, int d, int sign, bool wrap) const {
    int xs = x + sign * CX[d], ys = y + sign * CY[d], zs = z + sign * CZ[d];
    if (xs < 0 || xs >= nx) {
      if (!(wrap && per[0])) return -1;
      xs = (xs + nx) % nx;
    }
    if (ys < 0 || ys >= ny) {
      if (!(wrap && per[1])) return -1;
      ys = (ys + ny) % ny;
    }
    if (zs < 0 || zs >= nz) {
      if (!(wrap && per[2])) return -1;
      zs = (zs + nz) % nz;
    }
    return idx(xs, ys, zs);
  }

  // ---- link set ---------------------------------------------------------------------
  // Reference: nbr_lli has -1 off the domain, z included (Utilities.jl:559-569);
  // config: links follow the periodic axes.
  bool is_link(int x, int y, int z, int d) const {
    if (solid[idx(x, y, z)]) return false;
    int64_t nb = neighbour(x, y, z, d, +1, !ref());
    return nb >= 0 && solid[nb];
  }

  // ---- equilibria ---------------------------------------------------------------------
  // Reference feq in Collision.jl:233-237 / Initialization.jl:33-41 operation order.
  T feq_ref(int d, T r, T u, T v, T ww) const {
    T cu = T(CX[d]) * u + T(CY[d]) * v + T(CZ[d]) * ww;
    T cu2 = cu * cu;
    T u2 = u * u + v * v + ww * ww;
    return w[d] * r * (T(1) + cu * T(3) + T(0.5) * cu2 * T(9) - T(0.5) * u2 * T(3));
  }
  T feq_cfg(int d, T r, T u, T v, T ww) const {
    T cu = T(CX[d]) * u + T(CY[d]) * v + T(CZ[d]) * ww;
    T u2 = u * u + v * v + ww * ww;
    return w[d] * r * (T(1) + T(3) * cu + T(4.5) * cu * cu - T(1.5) * u2);
  }

  // ---- initial state --------------------------------------------------------------------
  int init_equilibrium(const double* r, const double* u, const double* v, const double* ww) {
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < N; i++) {
      T ri = r ? T(r[i]) : T(cfg.rho0);
      T ui = u ? T(u[i]) : T(0), vi = v ? T(v[i]) : T(0), wi = ww ? T(ww[i]) : T(0);
      for (int d = 0; d < Q; d++) {
        if (ref())
          S[d * N + i] = feq_ref(d, ri, ui, vi, wi);
        else
          S[d * N + i] = solid[i] ? T(0) : feq_cfg(d, ri, ui, vi, wi);
      }
    }
    if (ref()) compute_macros_ref();
    nstep = 0;
    force_hist.clear();
    return LBM_OK;
  }

  int set_populations(const double* f) {
    for (int64_t i = 0; i < (int64_t)Q * N; i++) S[i] = T(f[i]);
    if (ref()) compute_macros_ref();
    return LBM_OK;
  }

  // compute_macros!_gpu (ComputeMacro.jl:11-48): sequential sums over d = 1..q.
  void compute_macros_ref() {
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < N; i++) {
      T r = 0, mx = 0, my = 0, mz = 0;
      for (int d = 0; d < Q; d++) {
        T f = S[d * N + i];
        r += f;
        mx += f * T(CX[d]);
        my += f * T(CY[d]);
        mz += f * T(CZ[d]);
      }
      rho[i] = r;
      ux[i] = mx / r;
      uy[i] = my / r;
      uz[i] = mz / r;
    }
  }

  // ---- reference step --------------------------------------------------------------------
  void collide_ref() {
    // LBMParams fields are Float32 (Parameters.jl:8-47): round before promoting
    const T om_p = T((float)cfg.omega_p), om_m = T((float)cfg.omega_m);
    const bool trt = cfg.collision == LBM_COLL_TRT;
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < N; i++) {
      T r = rho[i], u = ux[i], v = uy[i], ww = uz[i];
      if (!trt) {
        // BGK_collision!_gpu, Collision.jl:229-238
        for (int d = 0; d < Q; d++) {
          T cu = T(CX[d]) * u + T(CY[d]) * v + T(CZ[d]) * ww;
          T cu2 = cu * cu;
          T u2 = u * u + v * v + ww * ww;
          T feq = w[d] * r * (T(1) + cu * T(3) + T(0.5) * cu2 * T(9) - T(0.5) * u2 * T(3));
          T fo = S[d * N + i];
          P[d * N + i] = fo - om_p * (fo - feq);
        }
      } else {
        // TRT_collision!_gpu, Collision.jl:136-170
        T u2 = u * u + v * v + ww * ww;
        for (int d = 0; d < Q; d++) {
          T fi = S[d * N + i], fo = S[OPP[d] * N + i];
          T cu = T(CX[d]) * u + T(CY[d]) * v + T(CZ[d]) * ww;
          T cu2 = cu * cu;
          T feq_p = w[d] * r * (T(1) + T(0.5) * cu2 * T(9) - T(0.5) * u2 * T(3));
          T feq_m = w[d] * r * (cu * T(3));
          T fp = T(0.5) * (fi + fo);
          T fm = T(0.5) * (fi - fo);
          T fpn = fp - om_p * (fp - feq_p);
          T fmn = fm - om_m * (fm - feq_m);
          P[d * N + i] = fpn + fmn;
        }
      }
    }
  }

  // Interpolated bounce-back of link (x, dir), solid at x + c_dir (lbm_config.solid_bc =
  // LBM_SOLID_IBB): IBB!_gpu (SolidBC.jl:253-338) with phi at the two ends of the link
  // x_b and x_b + c_dir, the wall point x_b + q c_dir, the fluid-side neighbour x_b - c_dir
  // for q <= 1/2 (across the periodic z axis as in streaming; outside the x/y range the
  // same-node branch) and q clamped to
  // [1e-4, 1 - 1e-4]; moving-wall bounce-back at the half-link point x_b + c_dir/2 when phi
  // does not change sign along the link.  Body at the half-step pose (Motion.jl:96-119),
  // lattice units, geometry in FP32; the interpolation in T.
  T ibb_value(int x, int y, int z, int dir) const {
    const lbm_body& b = bodies[moving_idx].b;
    const float h = (float)cfg.h;
    float ct = (float)pose_half.cos_theta, st = (float)pose_half.sin_theta;
    if (pose_half.cos_theta == 0.0 && pose_half.sin_theta == 0.0) {  // unset angle: 0
      ct = 1.0f;
      st = 0.0f;
    }
    const float xc = (float)pose_half.center[0], yc = (float)pose_half.center[1];
    auto phi = [&](float px, float py) -> float {
      if (b.kind == LBM_BODY_CYLINDER_Z) return phi_cylinder_f32(px, py, xc, yc, (float)b.radius / h);
      return phi_airfoil_f32(px, py, xc, yc, ct, st, (float)b.chord / h, (float)b.naca_m, (float)b.naca_p,
                             (float)b.naca_t, (float)b.x_int, (float)b.x_le_offset / h);
    };
    const float cxf = (float)CX[dir], cyf = (float)CY[dir];
    const float xb = (((float)(x + 1) - 0.5f) * h) / h;  // x_lli ./ h
    const float yb = (((float)(y + 1) - 0.5f) * h) / h;
    const float phib = phi(xb, yb);
    const float phis = phi(xb + cxf, yb + cyf);
    const float denom = phib - phis;
    const bool no_brkt = (phib <= 0.0f) || (phis >= 0.0f) || (std::fabs(denom) < 1e-8f);
    const float q = no_brkt ? 0.5f : std::min(std::max(phib / denom, 1e-4f), 1.0f - 1e-4f);
    const float xw = xb + q * cxf, yw = yb + q * cyf;
    const float rx = xw - (float)pose_half.center[0], ry = yw - (float)pose_half.center[1];
    const float uwx = (float)pose_half.vel[0] - (float)pose_half.omega[2] * ry;
    const float uwy = (float)pose_half.vel[1] + (float)pose_half.omega[2] * rx;
    const float cdu = cxf * uwx + cyf * uwy;
    const int64_t i = idx(x, y, z);
    const T corr = T(2) * w[dir] * rho[i] * T(cdu) * T(3);
    const T fdir = P[dir * N + i];
    if (no_brkt) return fdir - corr;
    const T tq = T(q);
    if (q <= 0.5f) {
      const int fx = x - CX[dir], fy = y - CY[dir], fz = (z - CZ[dir] + nz) % nz;  // z periodic
      if (fx >= 0 && fx < nx && fy >= 0 && fy < ny) {
        const T ff = P[dir * N + idx(fx, fy, fz)];
        return T(2) * tq * fdir + (T(1) - T(2) * tq) * ff - corr;
      }
    }
    const T fopp = P[OPP[dir] * N + i];
    return (T(0.5) / tq) * fdir + ((T(2) * tq - T(1)) / (T(2) * tq)) * fopp - corr;
  }

  void step_ref(double* F) {
    collide_ref();
    // streaming! (Streaming.jl:82-111) with stream_lidxs of build_stream_lists
    // (Utilities.jl:758-783) and the z-wrap copy of periodic_BC! (OtherBC.jl:65-82,
    // lists Utilities.jl:868-891).
#pragma omp parallel for schedule(static)
    for (int z = 0; z < nz; z++)
      for (int y = 0; y < ny; y++)
        for (int x = 0; x < nx; x++) {
          int64_t i = idx(x, y, z);
          for (int d = 0; d < Q; d++) {
            int sx = x - CX[d], sy = y - CY[d], sz = z - CZ[d];
            bool inx = sx >= 0 && sx < nx, iny = sy >= 0 && sy < ny, inz = sz >= 0 && sz < nz;
            int64_t src;
            if (inx && iny && inz)
              src = idx(sx, sy, sz);
            else if (!inz && inx && iny)
              src = idx(sx, sy, (sz + nz) % nz);  // periodic_BC!
            else
              src = i;  // x/y out of domain: same node, same direction
            S[d * N + i] = P[d * N + src];
          }
        }
    // SBB!_gpu (SolidBC.jl:160-210) over the link list, then MEA (MEA.jl:93-113).
    const float U = (float)pose_half.vel[0], V = (float)pose_half.vel[1];
    const float om = (float)pose_half.omega[2];
    const float xcl = (float)pose_half.center[0], ycl = (float)pose_half.center[1];
    const float h = (float)cfg.h;
    std::vector<double> Fz((size_t)nz * 6, 0.0);
#pragma omp parallel for schedule(static)
    for (int z = 0; z < nz; z++) {
      double acc[6] = {0, 0, 0, 0, 0, 0};
      for (int y = 0; y < ny; y++)
        for (int x = 0; x < nx; x++) {
          int64_t i = idx(x, y, z);
          if (solid[i]) continue;
          for (int dir = 0; dir < Q; dir++) {
            if (!is_link(x, y, z, dir)) continue;
            int opp = OPP[dir];
            T val;
            if (cfg.solid_bc == LBM_SOLID_IBB && moving_idx >= 0) {
              val = ibb_value(x, y, z, dir);
            } else if (sizeof(T) == 4) {
              float cx = (float)CX[dir], cy = (float)CY[dir];
              float xlat = (((float)(x + 1) - 0.5f) * h) / h;  // x_lli ./ h (MainCore.jl:199)
              float ylat = (((float)(y + 1) - 0.5f) * h) / h;
              float xw = xlat - 0.5f * cx, yw = ylat - 0.5f * cy;
              float rx = xw - xcl, ry = yw - ycl;
              float uwx = U - om * ry, uwy = V + om * rx;
              float cdu = cx * uwx + cy * uwy;
              float rw = (float)rho[i], wd = (float)w[dir];
              val = (T)((float)P[dir * N + i] - 2.0f * wd * rw * cdu * 3.0f);
            } else {
              double cx = CX[dir], cy = CY[dir];
              double xlat = (double)((((float)(x + 1) - 0.5f) * h) / h);
              double ylat = (double)((((float)(y + 1) - 0.5f) * h) / h);
              double xw = xlat - 0.5 * cx, yw = ylat - 0.5 * cy;
              double rx = xw - (double)xcl, ry = yw - (double)ycl;
              double uwx = (double)U - (double)om * ry, uwy = (double)V + (double)om * rx;
              double cdu = cx * uwx + cy * uwy;
              val = (T)((double)P[dir * N + i] - 2.0 * (double)w[dir] * (double)rho[i] * cdu * 3.0);
            }
            S[opp * N + i] = val;
          }
        }
      // faces: velocity entries first (inlet x=1, y=1, y=Ny), pressure (x=Nx) last.
      const T Ui = T((float)cfg.u_inf[0]), Vi = T((float)cfg.u_inf[1]), Wi = T((float)cfg.u_inf[2]);
      for (int y = 0; y < ny; y++)
        for (int x = 0; x < nx; x++) {
          int64_t i = idx(x, y, z);
          for (int pass = 0; pass < 2; pass++)
            for (int dir = 0; dir < Q; dir++) {
              bool vel = (x == 0 && CX[dir] > 0) || (y == 0 && CY[dir] > 0) ||
                         (y == ny - 1 && CY[dir] < 0);
              bool pres = (x == nx - 1 && CX[dir] < 0);
              int opp = OPP[dir];
              if (pass == 0 && vel) {
                // OtherBC.jl:139-148
                T cu = T(CX[dir]) * (-Ui) + T(CY[dir]) * (-Vi) + T(CZ[dir]) * (-Wi);
                S[dir * N + i] = P[opp * N + i] - T(2) * w[dir] * rho[i] * cu * T(3);
              }
              if (pass == 1 && pres) {
                // OtherBC.jl:153-165
                T cu = T(CX[dir]) * ux[i] + T(CY[dir]) * uy[i] + T(CZ[dir]) * uz[i];
                T cu2 = cu * cu;
                T uu2 = ux[i] * ux[i] + uy[i] * uy[i] + uz[i] * uz[i];
                S[dir * N + i] = -P[opp * N + i] +
                                 T(2) * w[dir] * rho[i] * (T(1) + T(0.5) * cu2 * T(9) - T(0.5) * uu2 * T(3));
              }
            }
        }
      // momentum exchange over the links of this plane
      for (int y = 0; y < ny; y++)
        for (int x = 0; x < nx; x++) {
          int64_t i = idx(x, y, z);
          if (solid[i]) continue;
          for (int dir = 0; dir < Q; dir++) {
            if (!is_link(x, y, z, dir)) continue;
            int opp = OPP[dir];
            double tmp = (double)P[dir * N + i] + (double)S[opp * N + i];
            double fx = tmp * CX[dir], fy = tmp * CY[dir], fz = tmp * CZ[dir];
            acc[0] += fx;
            acc[1] += fy;
            acc[2] += fz;
            // torque about the half-step centre (lattice units), planar lever arm
            double rxl = (double)(((float)(x + 1) - 0.5f) * h / h) - (double)xcl;
            double ryl = (double)(((float)(y + 1) - 0.5f) * h / h) - (double)ycl;
            double rzl = (z + 0.5) - pose_half.center[2];
            acc[3] += ryl * fz - rzl * fy;
            acc[4] += rzl * fx - rxl * fz;
            acc[5] += rxl * fy - ryl * fx;
          }
        }
      for (int k = 0; k < 6; k++) Fz[(size_t)z * 6 + k] = acc[k];
    }
    for (int z = 0; z < nz; z++)
      for (int k = 0; k < 6; k++) F[k] += Fz[(size_t)z * 6 + k];
    compute_macros_ref();
  }

  // ---- config step -------------------------------------------------------------------------
  void wall_velocity(double px, double py, double pz, double* uw) const {
    const lbm_pose& k = pose_half;
    double rx = px - k.center[0], ry = py - k.center[1], rz = pz - k.center[2];
    uw[0] = k.vel[0] + (k.omega[1] * rz - k.omega[2] * ry);
    uw[1] = k.vel[1] + (k.omega[2] * rx - k.omega[0] * rz);
    uw[2] = k.vel[2] + (k.omega[0] * ry - k.omega[1] * rx);
  }

  void step_cfg(double* F) {
    const T gx = T(cfg.accel[0]), gy = T(cfg.accel[1]), gz = T(cfg.accel[2]);
    const T om_p = T(cfg.omega_p), om_m = T(cfg.omega_m);
    const bool trt = cfg.collision == LBM_COLL_TRT;
    std::vector<T> rN(N), uN(N), vN(N), wN(N);
    // refill + collision of every fluid node
#pragma omp parallel for schedule(static)
    for (int z = 0; z < nz; z++)
      for (int y = 0; y < ny; y++)
        for (int x = 0; x < nx; x++) {
          int64_t i = idx(x, y, z);
          if (solid[i]) continue;
          T f[19];
          if (solid_prev[i]) {  // uncovered node: equilibrium at the body velocity
            double uw[3];
            wall_velocity(x + 0.5, y + 0.5, z + 0.5, uw);
            for (int d = 0; d < Q; d++) f[d] = feq_cfg(d, T(cfg.rho0), T(uw[0]), T(uw[1]), T(uw[2]));
          } else {
            for (int d = 0; d < Q; d++) f[d] = S[d * N + i];
          }
          T r = 0, jx = 0, jy = 0, jz = 0;
          for (int d = 0; d < Q; d++) {
            r += f[d];
            jx += f[d] * T(CX[d]);
            jy += f[d] * T(CY[d]);
            jz += f[d] * T(CZ[d]);
          }
          T u = jx / r + T(0.5) * gx, v = jy / r + T(0.5) * gy, ww = jz / r + T(0.5) * gz;
          T Fx = r * gx, Fy = r * gy, Fz = r * gz;
          T uF = u * Fx + v * Fy + ww * Fz;
          rN[i] = r;
          uN[i] = u;
          vN[i] = v;
          wN[i] = ww;
          T feq[19], Sd[19];
          for (int d = 0; d < Q; d++) {
            feq[d] = feq_cfg(d, r, u, v, ww);
            T cu = T(CX[d]) * u + T(CY[d]) * v + T(CZ[d]) * ww;
            T cF = T(CX[d]) * Fx + T(CY[d]) * Fy + T(CZ[d]) * Fz;
            Sd[d] = w[d] * (T(3) * (cF - uF) + T(9) * cu * cF);  // Guo source
          }
          if (!trt) {
            T fac = T(1) - T(0.5) * om_p;
            for (int d = 0; d < Q; d++) P[d * N + i] = f[d] - om_p * (f[d] - feq[d]) + fac * Sd[d];
          } else {
            T fac_p = T(1) - T(0.5) * om_p, fac_m = T(1) - T(0.5) * om_m;
            for (int d = 0; d < Q; d++) {
              int o = OPP[d];
              T fp = T(0.5) * (f[d] + f[o]), fm = T(0.5) * (f[d] - f[o]);
              T ep = T(0.5) * (feq[d] + feq[o]), em = T(0.5) * (feq[d] - feq[o]);
              T sp = T(0.5) * (Sd[d] + Sd[o]), sm = T(0.5) * (Sd[d] - Sd[o]);
              P[d * N + i] = f[d] - om_p * (fp - ep) - om_m * (fm - em) + fac_p * sp + fac_m * sm;
            }
          }
        }
    // pull streaming with boundary overrides
    std::vector<double> Fz((size_t)nz * 6, 0.0);
    int n3[3] = {nx, ny, nz};
#pragma omp parallel for schedule(static)
    for (int z = 0; z < nz; z++) {
      double acc[6] = {0, 0, 0, 0, 0, 0};
      for (int y = 0; y < ny; y++)
        for (int x = 0; x < nx; x++) {
          int64_t i = idx(x, y, z);
          if (solid[i]) {
            for (int d = 0; d < Q; d++) S[d * N + i] = T(0);
            continue;
          }
          int p[3] = {x, y, z};
          for (int d = 0; d < Q; d++) {
            int c[3] = {CX[d], CY[d], CZ[d]};
            int s[3];
            bool out[3];
            for (int a = 0; a < 3; a++) {
              s[a] = p[a] - c[a];
              out[a] = false;
              if (s[a] < 0 || s[a] >= n3[a]) {
                if (per[a])
                  s[a] = (s[a] + n3[a]) % n3[a];
                else
                  out[a] = true;
              }
            }
            int o = OPP[d];
            if (out[0] || out[1] || out[2]) {
              int face = out[0] ? (c[0] > 0 ? 0 : 1) : out[1] ? (c[1] > 0 ? 2 : 3) : (c[2] > 0 ? 4 : 5);
              const double* fu = cfg.face_u[face];
              T val;
              switch (cfg.face[face]) {
                case LBM_FACE_EQ_INLET:
                  val = feq_cfg(d, rN[i], T(fu[0]), T(fu[1]), T(fu[2]));
                  break;
                case LBM_FACE_OUTFLOW:
                  val = P[d * N + i];
                  break;
                case LBM_FACE_PRESSURE: {  // anti-bounce-back at rho0 with the node's velocity
                  T cu = T(CX[d]) * uN[i] + T(CY[d]) * vN[i] + T(CZ[d]) * wN[i];
                  T usq = uN[i] * uN[i] + vN[i] * vN[i] + wN[i] * wN[i];
                  val = -P[o * N + i] + T(2) * w[d] * T(cfg.rho0) * (T(1) + T(4.5) * cu * cu - T(1.5) * usq);
                  break;
                }
                default: {  // WALL: half-way bounce-back with wall velocity
                  T cdu = T(CX[o]) * T(fu[0]) + T(CY[o]) * T(fu[1]) + T(CZ[o]) * T(fu[2]);
                  val = P[o * N + i] - T(6) * w[o] * rN[i] * cdu;
                }
              }
              S[d * N + i] = val;
              continue;
            }
            int64_t src = idx(s[0], s[1], s[2]);
            if (solid[src]) {
              // link (i, o): moving-wall bounce-back at the half-way point
              double px = x + 0.5 + 0.5 * CX[o], py = y + 0.5 + 0.5 * CY[o], pz = z + 0.5 + 0.5 * CZ[o];
              double uw[3] = {0, 0, 0};
              if (moving[src]) wall_velocity(px, py, pz, uw);
              T cdu = T(CX[o]) * T(uw[0]) + T(CY[o]) * T(uw[1]) + T(CZ[o]) * T(uw[2]);
              T val = P[o * N + i] - T(6) * w[o] * rN[i] * cdu;
              S[d * N + i] = val;
              double tmp = (double)P[o * N + i] + (double)val;
              double fx = tmp * CX[o], fy = tmp * CY[o], fz = tmp * CZ[o];
              acc[0] += fx;
              acc[1] += fy;
              acc[2] += fz;
              double lc[3];
              lever_center(lc);
              double rx = px - lc[0], ry = py - lc[1], rz = pz - lc[2];
              acc[3] += ry * fz - rz * fy;
              acc[4] += rz * fx - rx * fz;
              acc[5] += rx * fy - ry * fx;
            } else {
              S[d * N + i] = P[d * N + src];
            }
          }
        }
      for (int k = 0; k < 6; k++) Fz[(size_t)z * 6 + k] = acc[k];
    }
    for (int z = 0; z < nz; z++)
      for (int k = 0; k < 6; k++) F[k] += Fz[(size_t)z * 6 + k];
    // after the step the node flags of this step are the "previous" flags
    std::copy(solid.begin(), solid.end(), solid_prev.begin());
  }

  int step(int nsteps) {
    for (int k = 0; k < nsteps; k++) {
      double F[6] = {0, 0, 0, 0, 0, 0};
      if (ref())
        step_ref(F);
      else
        step_cfg(F);
      nstep++;
      for (int j = 0; j < 6; j++) force_hist.push_back(F[j]);
    }
    return LBM_OK;
  }

  int get_macros(double* r, double* u, double* v, double* ww) const {
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < N; i++) {
      if (ref()) {
        if (r) r[i] = (double)rho[i];
        if (u) u[i] = (double)ux[i];
        if (v) v[i] = (double)uy[i];
        if (ww) ww[i] = (double)uz[i];
        continue;
      }
      if (solid[i]) {
        if (r) r[i] = 0;
        if (u) u[i] = 0;
        if (v) v[i] = 0;
        if (ww) ww[i] = 0;
        continue;
      }
      T rr = 0, jx = 0, jy = 0, jz = 0;
      for (int d = 0; d < Q; d++) {
        T f = S[d * N + i];
        rr += f;
        jx += f * T(CX[d]);
        jy += f * T(CY[d]);
        jz += f * T(CZ[d]);
      }
      if (r) r[i] = (double)rr;
      if (u) u[i] = (double)(jx / rr + T(0.5) * T(cfg.accel[0]));
      if (v) v[i] = (double)(jy / rr + T(0.5) * T(cfg.accel[1]));
      if (ww) ww[i] = (double)(jz / rr + T(0.5) * T(cfg.accel[2]));
    }
    return LBM_OK;
  }

  int get_flags(uint8_t* ms, uint8_t* mb) const {
    int lo[3], hi[3];
    const bool any = link_box(lo, hi);
#pragma omp parallel for schedule(static)
    for (int z = 0; z < nz; z++)
      for (int y = 0; y < ny; y++)
        for (int x = 0; x < nx; x++) {
          int64_t i = idx(x, y, z);
          if (ms) ms[i] = solid[i];
          if (mb) {
            bool hit = false;
            const bool in = any && x >= lo[0] && x <= hi[0] && y >= lo[1] && y <= hi[1] && z >= lo[2] && z <= hi[2];
            if (in && !solid[i])
              for (int d = 0; d < Q && !hit; d++) hit = is_link(x, y, z, d);
            mb[i] = hit;
          }
        }
    return LBM_OK;
  }

  int get_links(int32_t* ptr, int32_t* lidx, int8_t* dirs, int64_t cap, int64_t* nnz) const {
    int64_t k = 0;
    int lo[3], hi[3];
    const bool any = link_box(lo, hi);
    if (ptr) ptr[0] = 1;
    for (int z = 0; z < nz; z++)
      for (int y = 0; y < ny; y++)
        for (int x = 0; x < nx; x++) {
          int64_t i = idx(x, y, z);
          const bool in = any && x >= lo[0] && x <= hi[0] && y >= lo[1] && y <= hi[1] && z >= lo[2] && z <= hi[2];
          if (in)
            for (int d = 0; d < Q; d++)
              if (is_link(x, y, z, d)) {
                if (k < cap) {
                  if (lidx) lidx[k] = (int32_t)(i + 1);
                  if (dirs) dirs[k] = (int8_t)(d + 1);
                }
                k++;
              }
          if (ptr) ptr[i + 1] = (int32_t)(1 + k);
        }
    *nnz = k;
    return k > cap ? LBM_ERR_CAPACITY : LBM_OK;
  }

  int mass(double* out) const {
    double m = 0;
    for (int64_t i = 0; i < N; i++) {
      if (!ref() && solid[i]) continue;
      for (int d = 0; d < Q; d++) m += (double)S[d * N + i];
    }
    *out = m;
    return LBM_OK;
  }
};

}  // namespace

struct orc_sim {
  int prec;
  Sim<float>* f32 = nullptr;
  Sim<double>* f64 = nullptr;
  std::string err;
};

#define DISPATCH(s, call) ((s)->prec ? (s)->f64->call : (s)->f32->call)

extern "C" {

orc_sim* orc_create(const lbm_config* cfg, int32_t precision) {
  orc_sim* s = new orc_sim();
  s->prec = precision ? 1 : 0;
  int rc;
  if (s->prec) {
    s->f64 = new Sim<double>();
    rc = s->f64->init(cfg);
    if (rc) s->err = s->f64->err;
  } else {
    s->f32 = new Sim<float>();
    rc = s->f32->init(cfg);
    if (rc) s->err = s->f32->err;
  }
  if (rc) {
    fprintf(stderr, "orc_create: %s\n", s->err.c_str());
    delete s->f32;
    delete s->f64;
    delete s;
    return nullptr;
  }
  return s;
}

void orc_destroy(orc_sim* s) {
  if (!s) return;
  delete s->f32;
  delete s->f64;
  delete s;
}

const char* orc_last_error(const orc_sim* s) {
  if (!s) return "null";
  return s->prec ? s->f64->err.c_str() : s->f32->err.c_str();
}

int32_t orc_set_threads(int32_t n) {
#ifdef _OPENMP
  if (n > 0) omp_set_num_threads(n);
  return omp_get_max_threads();
#else
  (void)n;
  return 1;
#endif
}

int32_t orc_add_body(orc_sim* s, const lbm_body* b) { return DISPATCH(s, add_body(b)); }
int32_t orc_add_spheres(orc_sim* s, int32_t n, const double* xyzr) {
  return DISPATCH(s, add_spheres(n, xyzr));
}
int32_t orc_update_body(orc_sim* s, const lbm_pose* pn, const lbm_pose* ph) {
  return DISPATCH(s, update_body(pn, ph));
}
int32_t orc_init_equilibrium(orc_sim* s, const double* r, const double* u, const double* v,
                             const double* w) {
  return DISPATCH(s, init_equilibrium(r, u, v, w));
}
int32_t orc_set_populations(orc_sim* s, const double* f) { return DISPATCH(s, set_populations(f)); }
int32_t orc_step(orc_sim* s, int32_t n) { return DISPATCH(s, step(n)); }
int64_t orc_step_count(const orc_sim* s) { return s->prec ? s->f64->nstep : s->f32->nstep; }

int32_t orc_get_force(orc_sim* s, int64_t step, double out[6]) {
  const std::vector<double>& h = s->prec ? s->f64->force_hist : s->f32->force_hist;
  int64_t n = (int64_t)h.size() / 6;
  if (step < 1 || step > n) return LBM_ERR_ARG;
  for (int k = 0; k < 6; k++) out[k] = h[(size_t)(step - 1) * 6 + k];
  return LBM_OK;
}

int32_t orc_get_macros(orc_sim* s, double* r, double* u, double* v, double* w) {
  return DISPATCH(s, get_macros(r, u, v, w));
}

int32_t orc_get_populations(orc_sim* s, double* f) {
  if (s->prec) {
    auto& S = s->f64->S;
    for (size_t i = 0; i < S.size(); i++) f[i] = S[i];
  } else {
    auto& S = s->f32->S;
    for (size_t i = 0; i < S.size(); i++) f[i] = (double)S[i];
  }
  return LBM_OK;
}

int32_t orc_get_flags(orc_sim* s, uint8_t* ms, uint8_t* mb) { return DISPATCH(s, get_flags(ms, mb)); }
int32_t orc_get_links(orc_sim* s, int32_t* p, int32_t* l, int8_t* d, int64_t cap, int64_t* nnz) {
  return DISPATCH(s, get_links(p, l, d, cap, nnz));
}
int32_t orc_mass(orc_sim* s, double* out) { return DISPATCH(s, mass(out)); }

}  // extern "C"
