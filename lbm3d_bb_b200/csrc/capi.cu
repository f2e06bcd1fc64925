// capi.cu — the C ABI of liblbm3d.so (include/lbm3d.h): context, state machine,
// launches and the params.txt reader.
#include <cuda_runtime.h>

#include <algorithm>
#include <cctype>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "lbm_internal.cuh"
#include "lbm_kernels.h"

using namespace lbm;

namespace {

thread_local std::string g_error;

int set_global(int code, const char* fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof buf, fmt, ap);
  va_end(ap);
  g_error = buf;
  return code;
}

bool pose_equal(const lbm_pose& a, const lbm_pose& b) { return std::memcmp(&a, &b, sizeof(lbm_pose)) == 0; }

}  // namespace

struct lbm_ctx {
  lbm_config cfg{};
  int device = 0;
  cudaStream_t stream = nullptr;
  Grid g{};
  std::string err;
  bool ref = false;
  size_t elem = 4;  // bytes per stored population
  // config mode: AA array; reference mode: F[2], R[2]
  void* A = nullptr;
  void* F[2] = {nullptr, nullptr};
  void* R[2] = {nullptr, nullptr};
  int ri = 0;               // reference: buffer index of the current F/R
  bool ref_direct = false;  // reference: F[1-ri] holds S_n itself (no step since init)
  bool swapped = false;     // config: state in swapped layout (next phase odd)
  uint8_t* flags = nullptr;
  unsigned long long* links = nullptr;  // config mode: link words of NEAR nodes
  // TMA-staged step (config mode): per-tile boundary bits and the pipeline error word
  bool tma = false;
  int tma_tw = 0, tma_stages = 0;
  long long ntiles = 0;
  uint8_t* tiles = nullptr;
  bool tiles_dirty = true;
  int* d_err = nullptr;
  double* ring = nullptr;  // (cap + 1) force records of FORCE_RECORD doubles
  int ring_slots = 0;
  double* scratch = nullptr;  // 8 doubles
  long long nstep = 0;
  long long launches = 0;  // kernels this context has launched
  bool initialised = false;
  size_t bytes = 0;
  // bodies
  bool has_moving = false;
  lbm_body moving_body{};
  lbm_pose pose_bits_prev{}, pose_bits_cur{}, pose_last_step{}, pose_latest{};
  Kinematics kin_latest{}, kin_last_step{};
  double torque_center[3] = {0, 0, 0};
  bool any_body = false;
  // launch shape
  int bx = 0, by = 0;
  bool pair = false;  // FP16 pair kernel (see aa_pair_kernel)
  bool quad = false;  // FP16-deviation on the four-cell kernels
  bool xshuffle = false;  // FP32 odd phase on aa_pair_odd_kernel
  bool octo = false;  // FP16-deviation even phase on aa_octo_even_kernel
  bool quad_odd = false;  // FP16-deviation odd phase on aa_quad_odd_kernel

  int fail(int code, const char* fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    err = buf;
    return code;
  }
  int cuda(cudaError_t e, const char* what) {
    if (e == cudaSuccess) return LBM_OK;
    return fail(LBM_ERR_CUDA, "%s: %s", what, cudaGetErrorString(e));
  }
  dim3 block() const { return dim3((unsigned)bx, (unsigned)by, 1); }
  dim3 grid() const {
    return dim3((unsigned)((g.nx + bx - 1) / bx), (unsigned)((g.ny + by - 1) / by), (unsigned)g.nz);
  }
};

namespace {

void default_block(lbm_ctx* c) {
  // rows of the box across threadIdx.x; whole warps, at most 256 threads (the step
  // kernels' launch bound).  Rows that fit no such shape are padded to 32 lanes.
  const int nx = c->g.nx;
  int bx = nx <= 128 ? nx : 128;
  int by = std::max(1, 128 / bx);
  while ((bx * by) % 32 != 0 && bx * (by + 1) <= 256) by++;
  if ((bx * by) % 32 != 0) {
    bx = (nx + 31) / 32 * 32;
    by = std::max(1, 128 / bx);
  }
  const char* env = std::getenv("LBM3D_BLOCK");
  if (env) {
    int ex = 0, ey = 0;
    if (std::sscanf(env, "%d,%d", &ex, &ey) == 2 && ex > 0 && ey > 0 && ex * ey <= 1024 && (ex * ey) % 32 == 0) {
      bx = ex;
      by = ey;
    }
  }
  c->bx = bx;
  c->by = by;
}

BodyDev to_dev(const lbm_ctx* c, const lbm_body& b, const lbm_pose* pose) {
  BodyDev d{};
  d.kind = b.kind;
  d.radius = b.radius;
  for (int k = 0; k < 3; k++) d.semi[k] = b.semi[k];
  d.chord = b.chord;
  d.naca_m = b.naca_m;
  d.naca_p = b.naca_p;
  d.naca_t = b.naca_t;
  d.x_int = b.x_int;
  d.x_le_offset = b.x_le_offset;
  d.h = c->cfg.h;
  const double* rot = b.rot;
  double ident[9] = {1, 0, 0, 0, 1, 0, 0, 0, 1};
  if (pose) {
    for (int k = 0; k < 3; k++) d.center[k] = pose->center[k];
    d.cos_t = pose->cos_theta;
    d.sin_t = pose->sin_theta;
    rot = pose->rot;
  } else {
    for (int k = 0; k < 3; k++) d.center[k] = b.center[k];
  }
  bool zero = true;
  for (int k = 0; k < 9; k++) zero = zero && rot[k] == 0.0;
  for (int k = 0; k < 9; k++) d.rot[k] = zero ? ident[k] : rot[k];
  if (!pose) {
    d.cos_t = d.rot[0];
    d.sin_t = d.rot[3];
  }
  return d;
}

// Lattice-index bounding box of a body at a pose, dilated by `pad` cells.
Box body_box(const lbm_ctx* c, const lbm_body& b, const double* center, int pad) {
  Box bx{};
  const int n3[3] = {c->g.nx, c->g.ny, c->g.nz};
  double rad[3];
  double cl[3];
  const bool planar = (b.kind == LBM_BODY_CYLINDER_Z || b.kind == LBM_BODY_NACA_Z);
  const double h = c->cfg.h;
  double r = 0;
  switch (b.kind) {
    case LBM_BODY_CYLINDER_Z: r = b.radius / h; break;
    case LBM_BODY_NACA_Z: r = (std::fabs(b.chord) + std::fabs(b.x_le_offset)) / h + 1.0; break;
    case LBM_BODY_SPHERE: r = b.radius; break;
    case LBM_BODY_ELLIPSOID: r = std::max(b.semi[0], std::max(b.semi[1], b.semi[2])); break;
  }
  for (int a = 0; a < 3; a++) {
    rad[a] = r;
    // node (ix) sits at lattice coordinate ix + 0.5; planar shapes use physical units / h
    cl[a] = planar ? center[a] / h - 0.5 : center[a] - 0.5;
  }
  for (int a = 0; a < 3; a++) {
    if (planar && a == 2) {
      bx.lo[a] = 0;
      bx.hi[a] = n3[a] - 1;
      continue;
    }
    bx.lo[a] = (int)std::floor(cl[a] - rad[a]) - pad;
    bx.hi[a] = (int)std::ceil(cl[a] + rad[a]) + pad;
  }
  return bx;
}

Box box_union(const Box& a, const Box& b) {
  Box r{};
  for (int k = 0; k < 3; k++) {
    r.lo[k] = std::min(a.lo[k], b.lo[k]);
    r.hi[k] = std::max(a.hi[k], b.hi[k]);
  }
  return r;
}

// Clamp to the domain; periodic axes keep unwrapped ranges shorter than n.
bool box_clamp(const lbm_ctx* c, Box& b) {
  const int n3[3] = {c->g.nx, c->g.ny, c->g.nz};
  for (int a = 0; a < 3; a++) {
    if (c->g.per[a]) {
      if (b.hi[a] - b.lo[a] + 1 >= n3[a]) {
        b.lo[a] = 0;
        b.hi[a] = n3[a] - 1;
      }
    } else {
      b.lo[a] = std::max(b.lo[a], 0);
      b.hi[a] = std::min(b.hi[a], n3[a] - 1);
      if (b.hi[a] < b.lo[a]) return false;
    }
  }
  return true;
}

Box dilate(Box b, int k) {
  for (int a = 0; a < 3; a++) {
    b.lo[a] -= k;
    b.hi[a] += k;
  }
  return b;
}

Box full_box(const lbm_ctx* c) {
  Box b{};
  b.lo[0] = b.lo[1] = b.lo[2] = 0;
  b.hi[0] = c->g.nx - 1;
  b.hi[1] = c->g.ny - 1;
  b.hi[2] = c->g.nz - 1;
  return b;
}

// Bring the flag bytes to: SOLID = flags at pose_latest, SOLID_PREV = flags at
// pose_last_step (and NEAR consistent with both).
int sync_flags(lbm_ctx* c) {
  if (!c->has_moving) return LBM_OK;
  if (pose_equal(c->pose_bits_prev, c->pose_last_step) && pose_equal(c->pose_bits_cur, c->pose_latest))
    return LBM_OK;
  const lbm_body& b = c->moving_body;
  Box r = body_box(c, b, c->pose_bits_prev.center, 2);
  r = box_union(r, body_box(c, b, c->pose_bits_cur.center, 2));
  r = box_union(r, body_box(c, b, c->pose_last_step.center, 2));
  r = box_union(r, body_box(c, b, c->pose_latest.center, 2));
  Box rn = dilate(r, 1);
  if (box_clamp(c, r)) {
    FlagParams p{};
    p.g = c->g;
    p.mode = c->cfg.mode;
    p.box = r;
    p.body = to_dev(c, b, &c->pose_latest);
    p.body_prev = to_dev(c, b, &c->pose_last_step);
    p.has_moving = 1;
    c->launches++;
    int rc = c->cuda(geo_launch_moving(p, c->flags, c->stream), "moving-body flags");
    if (rc) return rc;
  }
  if (box_clamp(c, rn)) {
    c->launches++;
    int rc = c->cuda(geo_launch_near(c->g, c->cfg.mode, rn, c->flags, c->links, c->stream), "near flags");
    if (rc) return rc;
  }
  c->pose_bits_prev = c->pose_last_step;
  c->pose_bits_cur = c->pose_latest;
  c->tiles_dirty = true;
  return LBM_OK;
}

// Kinematics of a pose (lattice units as given by the caller).
Kinematics kin_of(const lbm_pose& p) {
  Kinematics k{};
  for (int a = 0; a < 3; a++) {
    k.center[a] = p.center[a];
    k.vel[a] = p.vel[a];
    k.omega[a] = p.omega[a];
  }
  // an unset angle (cos = sin = 0) is angle 0
  const bool unset = p.cos_theta == 0.0 && p.sin_theta == 0.0;
  k.cos_t = unset ? 1.0 : p.cos_theta;
  k.sin_t = unset ? 0.0 : p.sin_theta;
  return k;
}

// Device copy of an optional host/device array of n doubles.
struct DevBuf {
  void* p = nullptr;
  ~DevBuf() {
    if (p) cudaFree(p);
  }
};

int stage_in(lbm_ctx* c, const void* src, size_t bytes, int where, DevBuf& buf, const void** out) {
  if (!src) {
    *out = nullptr;
    return LBM_OK;
  }
  if (where == LBM_DEVICE) {
    *out = src;
    return LBM_OK;
  }
  int rc = c->cuda(cudaMalloc(&buf.p, bytes), "cudaMalloc(staging)");
  if (rc) return rc;
  rc = c->cuda(cudaMemcpyAsync(buf.p, src, bytes, cudaMemcpyHostToDevice, c->stream), "H2D staging");
  if (rc) return rc;
  *out = buf.p;
  return LBM_OK;
}

RefParams ref_params(const lbm_ctx* c, const Kinematics& kin, uint8_t solid_bit) {
  RefParams p{};
  p.g = c->g;
  p.omega_p = (float)c->cfg.omega_p;
  p.omega_m = (float)c->cfg.omega_m;
  p.U = (float)c->cfg.u_inf[0];
  p.V = (float)c->cfg.u_inf[1];
  p.W = (float)c->cfg.u_inf[2];
  p.h = (float)c->cfg.h;
  p.kin = kin;
  p.solid_bit = solid_bit;
  p.compute_force = 0;
  p.solid_bc = c->cfg.solid_bc;
  if (c->cfg.solid_bc == LBM_SOLID_IBB && c->has_moving) {
    // the body as IBB!_gpu sees it: half-step pose, lattice units (Motion.jl:96-119)
    const lbm_body& b = c->moving_body;
    const float h = (float)c->cfg.h;
    IbbGeom& q = p.ibb;
    q.shape = b.kind;
    q.xc = (float)kin.center[0];
    q.yc = (float)kin.center[1];
    q.ct = (float)kin.cos_t;
    q.st = (float)kin.sin_t;
    q.R = (float)b.radius / h;
    q.chord = (float)b.chord / h;
    q.x_le = (float)b.x_le_offset / h;
    q.m = (float)b.naca_m;
    q.p = (float)b.naca_p;
    q.t = (float)b.naca_t;
    q.x_int = (float)b.x_int;
  }
  return p;
}

ReadParams read_params(const lbm_ctx* c) {
  ReadParams p{};
  p.g = c->g;
  p.rho0 = c->cfg.rho0;
  p.swapped = c->swapped ? 1 : 0;
  p.solid_bit = F_SOLID_PREV;
  for (int a = 0; a < 3; a++) p.gacc[a] = c->cfg.accel[a];
  return p;
}

bool is_ref_fp64(const lbm_ctx* c) { return c->cfg.storage == LBM_STORE_FP64; }

// Export of S_n / macros through `out` (device pointers).
int export_state(lbm_ctx* c, const ExportOut& out) {
  int rc = sync_flags(c);
  if (rc) return rc;
  if (c->ref) {
    RefParams p = ref_params(c, c->kin_last_step, F_SOLID_PREV);
    return c->cuda(ref_launch_export(is_ref_fp64(c), p, c->F[1 - c->ri], c->R[1 - c->ri], c->ref_direct ? 1 : 0,
                                     c->flags, out, nullptr, c->grid(), c->block(), c->stream),
                   "export");
  }
  return c->cuda(aa_launch_export(c->cfg.storage, read_params(c), c->A, c->flags, out, c->grid(), c->block(),
                                  c->stream),
                 "export");
}

int reduce_state(lbm_ctx* c, double out[2]) {
  int rc = sync_flags(c);
  if (rc) return rc;
  rc = c->cuda(cudaMemsetAsync(c->scratch, 0, 8 * sizeof(double), c->stream), "memset");
  if (rc) return rc;
  if (c->ref) {
    RefParams p = ref_params(c, c->kin_last_step, F_SOLID_PREV);
    ExportOut none{};
    rc = c->cuda(ref_launch_export(is_ref_fp64(c), p, c->F[1 - c->ri], c->R[1 - c->ri], c->ref_direct ? 1 : 0,
                                   c->flags, none, c->scratch, c->grid(), c->block(), c->stream),
                 "reduce");
  } else {
    rc = c->cuda(aa_launch_reduce(c->cfg.storage, read_params(c), c->A, c->flags, c->scratch, c->grid(),
                                  c->block(), c->stream),
                 "reduce");
  }
  if (rc) return rc;
  double h[6];
  rc = c->cuda(cudaMemcpyAsync(h, c->scratch, 6 * sizeof(double), cudaMemcpyDeviceToHost, c->stream), "D2H");
  if (rc) return rc;
  rc = c->cuda(cudaStreamSynchronize(c->stream), "sync");
  if (rc) return rc;
  out[0] = h[0];
  out[1] = h[1];
  return LBM_OK;
}

// Parameter block of the config-mode step for one phase (odd: the populations are in
// the swapped layout).  force/zero_next are left for the caller.
void fill_aa_params(const lbm_ctx* c, AAParams& p, bool odd) {
  p = AAParams{};
  p.g = c->g;
  for (int f = 0; f < 6; f++) {
    p.face_kind[f] = c->cfg.face[f];
    for (int a = 0; a < 3; a++) p.face_u[f][a] = c->cfg.face_u[f][a];
  }
  p.omega_p = c->cfg.omega_p;
  p.omega_m = c->cfg.omega_m;
  p.rho0 = c->cfg.rho0;
  for (int a = 0; a < 3; a++) p.gacc[a] = c->cfg.accel[a];
  p.kin = c->kin_latest;
  if (!c->has_moving)
    for (int a = 0; a < 3; a++) p.kin.center[a] = c->torque_center[a];
  p.compute_force = c->cfg.compute_force ? 1 : 0;
  p.links = c->links;
  const long long nx = c->g.nx, nxy = (long long)c->g.nx * c->g.ny, pl = c->g.plane;
  for (int d = 0; d < 19; d++) {
    const long long nb = cx(d) + nx * cy(d) + nxy * cz(d);
    if (!odd) {  // even phase: own slots
      p.off_rd[d] = d * pl;
      p.off_wr[d] = d * pl;
    } else {  // odd phase: pull from x - c_d (slot opp(d)), push to x + c_d (slot d)
      p.off_rd[d] = opp(d) * pl - nb;
      p.off_wr[d] = d * pl + nb;
    }
    p.offb_rd[d] = p.off_rd[d] * c->elem;
    p.offb_wr[d] = p.off_wr[d] * c->elem;
  }
}

bool has_force(const lbm_ctx* c) { return c->cfg.accel[0] != 0.0 || c->cfg.accel[1] != 0.0 || c->cfg.accel[2] != 0.0; }
// step kernels' force mode: 0 none, 1 general, 2 acceleration along x only (the y and z
// source terms are exact zeros and are skipped; FP16-deviation storage, where the
// issue-bound kernels gain 4 %)
int force_mode(const lbm_ctx* c) {
  if (!has_force(c)) return 0;
  const bool x_only = c->cfg.accel[1] == 0.0 && c->cfg.accel[2] == 0.0;
  return x_only && c->cfg.storage == LBM_STORE_FP16DEV ? 2 : 1;
}
bool has_faces(const lbm_ctx* c) { return !(c->g.per[0] && c->g.per[1] && c->g.per[2]); }
bool has_halo(const lbm_ctx* c) {
  return !c->ref && (c->cfg.face[4] == LBM_FACE_HALO || c->cfg.face[5] == LBM_FACE_HALO);
}
// periodic x and y, halo faces on both z ends: no face node outside the ghost planes, so
// the step kernels without face handling (and the pair kernel) serve it, skipping the
// ghost planes block by block
bool halo_only(const lbm_ctx* c) {
  return !c->ref && c->g.per[0] && c->g.per[1] && c->cfg.face[4] == LBM_FACE_HALO &&
         c->cfg.face[5] == LBM_FACE_HALO;
}

int near_full(lbm_ctx* c) {
  c->tiles_dirty = true;
  Box f = full_box(c);
  return c->cuda(geo_launch_near(c->g, c->cfg.mode, f, c->flags, c->links, c->stream), "near flags");
}

// ---- params.txt ---------------------------------------------------------------------
std::string strip(const std::string& s) {
  size_t a = 0, b = s.size();
  while (a < b && std::isspace((unsigned char)s[a])) a++;
  while (b > a && std::isspace((unsigned char)s[b - 1])) b--;
  return s.substr(a, b - a);
}

// ^KEY:\s*\|?\s*(token) where token chars satisfy `ok`
bool key_token(const std::string& line, size_t klen, bool (*ok)(char), std::string* tok) {
  size_t i = klen;
  while (i < line.size() && std::isspace((unsigned char)line[i])) i++;
  if (i < line.size() && line[i] == '|') i++;
  while (i < line.size() && std::isspace((unsigned char)line[i])) i++;
  size_t j = i;
  while (j < line.size() && ok(line[j])) j++;
  if (j == i) return false;
  *tok = line.substr(i, j - i);
  return true;
}
bool ok_ident(char ch) { return std::isalnum((unsigned char)ch) || ch == '_' || ch == '+' || ch == '-'; }
bool ok_alpha(char ch) { return std::isalpha((unsigned char)ch) != 0; }

// leftmost match of [+-]?\d+(?:\.\d*)?(?:[eE][+-]?\d+)?
bool first_number(const std::string& s, std::string* out) {
  const size_t n = s.size();
  for (size_t st = 0; st < n; st++) {
    size_t i = st;
    if (s[i] == '+' || s[i] == '-') i++;
    if (i >= n || !std::isdigit((unsigned char)s[i])) continue;
    while (i < n && std::isdigit((unsigned char)s[i])) i++;
    if (i < n && s[i] == '.') {
      i++;
      while (i < n && std::isdigit((unsigned char)s[i])) i++;
    }
    if (i < n && (s[i] == 'e' || s[i] == 'E')) {
      size_t k = i + 1;
      if (k < n && (s[k] == '+' || s[k] == '-')) k++;
      if (k < n && std::isdigit((unsigned char)s[k])) {
        while (k < n && std::isdigit((unsigned char)s[k])) k++;
        i = k;
      }
    }
    *out = s.substr(st, i - st);
    return true;
  }
  return false;
}

bool to_int(float v, int32_t* out) {
  if (!std::isfinite(v) || std::floor(v) != v) return false;
  *out = (int32_t)v;
  return true;
}

}  // namespace

// =========================================================================================
extern "C" {

int32_t lbm_abi_version(void) { return LBM3D_ABI_VERSION; }

const char* lbm_status_string(int32_t s) {
  switch (s) {
    case LBM_OK: return "ok";
    case LBM_ERR_ARG: return "invalid argument";
    case LBM_ERR_CUDA: return "CUDA error";
    case LBM_ERR_STATE: return "invalid state";
    case LBM_ERR_UNSUPPORTED: return "unsupported";
    case LBM_ERR_PARSE: return "parse error";
    case LBM_ERR_NUMERIC: return "non-finite populations";
    case LBM_ERR_CAPACITY: return "capacity exceeded";
    case LBM_ERR_TIMEOUT: return "a bounded device wait gave up";
  }
  return "unknown status";
}

const char* lbm_global_error(void) { return g_error.c_str(); }

int32_t lbm_lattice(int32_t q, int8_t* ocx, int8_t* ocy, int8_t* ocz, float* w, int8_t* oop) {
  if (q != 19 && q != 27) return set_global(LBM_ERR_UNSUPPORTED, "q=19 or q=27 (got %d)", q);
  for (int d = 0; d < q; d++) {
    if (ocx) ocx[d] = (int8_t)(q == 19 ? cx(d) : cx27(d));
    if (ocy) ocy[d] = (int8_t)(q == 19 ? cy(d) : cy27(d));
    if (ocz) ocz[d] = (int8_t)(q == 19 ? cz(d) : cz27(d));
    if (w) w[d] = q == 19 ? wgt<float>(d) : wgt27<float>(d);
    if (oop) oop[d] = (int8_t)(d == q - 1 ? d : (d ^ 1));
  }
  return LBM_OK;
}

int32_t lbm_read_params(const char* path, lbm_params* out) {
  if (!path || !out) return set_global(LBM_ERR_ARG, "null argument");
  FILE* fp = std::fopen(path, "rb");
  if (!fp) return set_global(LBM_ERR_PARSE, "cannot open %s", path);
  std::string content;
  char buf[4096];
  size_t n;
  while ((n = std::fread(buf, 1, sizeof buf, fp)) > 0) content.append(buf, n);
  std::fclose(fp);
  std::vector<float> values;
  std::string bc, coll, naca;
  bool have_bc = false, have_coll = false, have_naca = false;
  int shape = 1;
  size_t pos = 0;
  while (pos <= content.size()) {
    size_t e = content.find('\n', pos);
    if (e == std::string::npos) e = content.size();
    const std::string raw = content.substr(pos, e - pos);
    pos = e + 1;
    const std::string line = strip(raw);
    if (line.empty() || line[0] == '#') {
      if (e == content.size()) break;
      continue;
    }
    std::string tok;
    if (line.compare(0, 3, "BC:") == 0) {
      if (!key_token(line, 3, ok_ident, &tok)) return set_global(LBM_ERR_PARSE, "Could not parse BC from: %s", raw.c_str());
      bc = tok;
      have_bc = true;
    } else if (line.compare(0, 5, "Coll:") == 0) {
      if (!key_token(line, 5, ok_ident, &tok)) return set_global(LBM_ERR_PARSE, "Could not parse Coll from: %s", raw.c_str());
      coll = tok;
      have_coll = true;
    } else if (line.compare(0, 6, "Shape:") == 0) {
      if (!key_token(line, 6, ok_alpha, &tok)) return set_global(LBM_ERR_PARSE, "Could not parse Shape from: %s", raw.c_str());
      for (auto& ch : tok) ch = (char)std::toupper((unsigned char)ch);
      if (tok != "CYL" && tok != "AIR") return set_global(LBM_ERR_PARSE, "Shape must be CYL or AIR, got %s", tok.c_str());
      shape = tok == "CYL" ? 1 : 2;
    } else if (line.compare(0, 5, "NACA:") == 0) {
      std::string digits;
      size_t i = 5;
      while (i < line.size() && std::isspace((unsigned char)line[i])) i++;
      if (i < line.size() && line[i] == '|') i++;
      while (i < line.size() && std::isspace((unsigned char)line[i])) i++;
      size_t j = i;
      while (j < line.size() && j - i < 4 && std::isdigit((unsigned char)line[j])) j++;
      if (j - i != 4)
        return set_global(LBM_ERR_PARSE, "Could not parse NACA code (expect 4 digits) from: %s", raw.c_str());
      naca = line.substr(i, 4);
      have_naca = true;
    } else {
      std::string num;
      if (!first_number(line, &num)) return set_global(LBM_ERR_PARSE, "Could not find a number in: %s", raw.c_str());
      values.push_back(std::strtof(num.c_str(), nullptr));
    }
    if (e == content.size()) break;
  }
  if (values.size() != 19)
    return set_global(LBM_ERR_PARSE, "Expected 19 numeric parameters, got %d.", (int)values.size());
  if (!have_bc) return set_global(LBM_ERR_PARSE, "Missing BC line in input file!");
  if (!have_coll) coll = "BGK";
  if (shape == 2 && !have_naca) naca = "0012";
  lbm_params p{};
  if (!to_int(values[0], &p.Nx) || !to_int(values[1], &p.Ny) || !to_int(values[2], &p.Nz) ||
      !to_int(values[9], &p.q) || !to_int(values[17], &p.n_max) || !to_int(values[18], &p.n_save))
    return set_global(LBM_ERR_PARSE, "InexactError: an integer parameter is not integral");
  p.h = values[3];
  p.R = values[4];
  p.x_c = values[5];
  p.y_c = values[6];
  p.theta0 = values[7] * (3.14159265358979323846f / 180.0f);  // deg2rad(::Float32)
  p.chord = values[8];
  p.Re = values[10];
  p.U_inf = values[11];
  p.V_inf = values[12];
  p.W_inf = values[13];
  p.rho_inf = values[14];
  p.dt = values[15];
  p.Lambda = values[16];
  // LBMParams constructor (Parameters.jl:62-72), FP32
  const float L = ((shape == 1) ? (2.0f * p.R) : p.chord) / p.h;
  p.nu = (p.U_inf * L) / p.Re;
  const float tau_p = 0.5f + 3.0f * p.nu;
  const float tau_m = 0.5f + p.Lambda / (tau_p - 0.5f);
  p.omega_p = 1.0f / tau_p;
  p.omega_m = 1.0f / tau_m;
  std::snprintf(p.bc, sizeof p.bc, "%s", bc.c_str());
  std::snprintf(p.coll, sizeof p.coll, "%s", coll.c_str());
  p.shape = shape;
  std::snprintf(p.naca_code, sizeof p.naca_code, "%s", naca.c_str());
  *out = p;
  return LBM_OK;
}

int32_t lbm_create(const lbm_config* cfg, int32_t device, lbm_ctx** out) {
  if (!cfg || !out) return set_global(LBM_ERR_ARG, "null argument");
  *out = nullptr;
  if (cfg->q != 19 && !(cfg->q == 27 && cfg->mode == LBM_MODE_REFERENCE))
    return set_global(LBM_ERR_UNSUPPORTED, "q=%d: D3Q19, or D3Q27 in reference mode", cfg->q);
  if (cfg->solid_bc != LBM_SOLID_SBB && cfg->solid_bc != LBM_SOLID_IBB)
    return set_global(LBM_ERR_ARG, "solid_bc %d is not LBM_SOLID_SBB or LBM_SOLID_IBB", cfg->solid_bc);
  if (cfg->solid_bc == LBM_SOLID_IBB && cfg->mode != LBM_MODE_REFERENCE)
    return set_global(LBM_ERR_UNSUPPORTED, "the interpolated bounce-back is a reference-mode rule");
  if (cfg->nx < 2 || cfg->ny < 2 || cfg->nz < 1) return set_global(LBM_ERR_ARG, "bad dimensions %dx%dx%d", cfg->nx, cfg->ny, cfg->nz);
  if ((long long)cfg->nx * cfg->ny * cfg->nz >= (1LL << 31))
    return set_global(LBM_ERR_ARG, "more than 2^31-1 nodes");
  if (cfg->mode != LBM_MODE_REFERENCE && cfg->mode != LBM_MODE_CONFIG) return set_global(LBM_ERR_ARG, "bad mode");
  if (cfg->collision != LBM_COLL_BGK && cfg->collision != LBM_COLL_TRT) return set_global(LBM_ERR_ARG, "bad collision");
  if (cfg->storage < LBM_STORE_FP32 || cfg->storage > LBM_STORE_FP16DEV) return set_global(LBM_ERR_ARG, "bad storage");
  if (cfg->mode == LBM_MODE_REFERENCE && cfg->storage == LBM_STORE_FP16DEV)
    return set_global(LBM_ERR_UNSUPPORTED, "reference mode stores FP32 or FP64");
  if (!(cfg->omega_p > 0.0 && cfg->omega_p < 2.0)) return set_global(LBM_ERR_ARG, "omega_p must lie in (0, 2)");
  if (cfg->collision == LBM_COLL_TRT && !(cfg->omega_m > 0.0 && cfg->omega_m < 2.0))
    return set_global(LBM_ERR_ARG, "omega_m must lie in (0, 2)");
  if (cfg->mode == LBM_MODE_CONFIG) {
    for (int a = 0; a < 3; a++) {
      const bool p0 = cfg->face[2 * a] == LBM_FACE_PERIODIC, p1 = cfg->face[2 * a + 1] == LBM_FACE_PERIODIC;
      if (p0 != p1) return set_global(LBM_ERR_ARG, "axis %d: both faces periodic or neither", a);
      for (int s = 0; s < 2; s++) {
        if (cfg->face[2 * a + s] < LBM_FACE_PERIODIC || cfg->face[2 * a + s] > LBM_FACE_HALO)
          return set_global(LBM_ERR_ARG, "bad face kind");
        if (cfg->face[2 * a + s] == LBM_FACE_HALO && a != 2) return set_global(LBM_ERR_ARG, "halo faces are z faces");
      }
    }
    if ((cfg->face[4] == LBM_FACE_HALO || cfg->face[5] == LBM_FACE_HALO) && cfg->nz < 3)
      return set_global(LBM_ERR_ARG, "a slab with halo faces needs nz >= 3");
  }
  lbm_ctx* c = new lbm_ctx();
  c->cfg = *cfg;
  if (c->cfg.h == 0.0) c->cfg.h = 1.0;
  if (c->cfg.rho0 == 0.0) c->cfg.rho0 = 1.0;
  if (c->cfg.force_history < 1) c->cfg.force_history = 1;
  c->device = device;
  c->ref = cfg->mode == LBM_MODE_REFERENCE;
  c->g.nx = cfg->nx;
  c->g.ny = cfg->ny;
  c->g.nz = cfg->nz;
  if (c->ref) {
    c->g.per[0] = c->g.per[1] = 0;
    c->g.per[2] = 1;
  } else {
    for (int a = 0; a < 3; a++) c->g.per[a] = cfg->face[2 * a] == LBM_FACE_PERIODIC ? 1 : 0;
  }
  c->g.N = (long long)cfg->nx * cfg->ny * cfg->nz;
  c->g.plane = (c->g.N + 127) / 128 * 128;  // 256-byte aligned planes for every storage
  c->g.q = cfg->q;
  c->elem = cfg->storage == LBM_STORE_FP64 ? 8 : (cfg->storage == LBM_STORE_FP16DEV ? 2 : 4);
  default_block(c);
  auto bail = [&](int rc) {
    set_global(rc, "%s", c->err.c_str());
    lbm_destroy(c);
    return rc;
  };
  if (c->cuda(cudaSetDevice(device), "cudaSetDevice")) return bail(LBM_ERR_CUDA);
  const size_t pop = (size_t)cfg->q * c->g.plane * c->elem;
  const size_t fl = (size_t)((c->g.N + 3) / 4 * 4);
  if (c->ref) {
    const size_t rb = (size_t)4 * c->g.N * c->elem;
    for (int k = 0; k < 2; k++) {
      if (c->cuda(cudaMalloc(&c->F[k], pop), "cudaMalloc(populations)")) return bail(LBM_ERR_CUDA);
      if (c->cuda(cudaMalloc(&c->R[k], rb), "cudaMalloc(macros)")) return bail(LBM_ERR_CUDA);
      c->bytes += pop + rb;
    }
  } else {
    if (c->cuda(cudaMalloc(&c->A, pop), "cudaMalloc(populations)")) return bail(LBM_ERR_CUDA);
    c->bytes += pop;
  }
  if (c->cuda(cudaMalloc(&c->flags, fl), "cudaMalloc(flags)")) return bail(LBM_ERR_CUDA);
  if (!c->ref) {
    if (c->cuda(cudaMalloc(&c->links, (size_t)c->g.N * 8), "cudaMalloc(links)")) return bail(LBM_ERR_CUDA);
    if (c->cuda(cudaMemset(c->links, 0, (size_t)c->g.N * 8), "memset links")) return bail(LBM_ERR_CUDA);
    c->bytes += (size_t)c->g.N * 8;
  }
  c->ring_slots = c->cfg.force_history + 1;
  const size_t ring_bytes = (size_t)c->ring_slots * FORCE_RECORD * sizeof(double);
  if (c->cuda(cudaMalloc(&c->ring, ring_bytes), "cudaMalloc(force ring)")) return bail(LBM_ERR_CUDA);
  if (c->cuda(cudaMalloc(&c->scratch, 8 * sizeof(double)), "cudaMalloc(scratch)")) return bail(LBM_ERR_CUDA);
  if (c->cuda(cudaMalloc(&c->d_err, sizeof(int)), "cudaMalloc(err)")) return bail(LBM_ERR_CUDA);
  if (c->cuda(cudaMemset(c->d_err, 0, sizeof(int)), "memset err")) return bail(LBM_ERR_CUDA);
  // TMA-staged step (opt-in with LBM3D_TMA=1): rows split into 128-cell tiles with
  // 16-byte aligned segments.  On B200 the bulk-copy pipeline measured below the
  // direct kernel (a pure data-movement probe of this 19-plane pattern reached
  // 6.1 TB/s through TMA against 6.8 TB/s with plain coalesced loads), so the
  // direct kernel is the default.
  {
    const char* on = std::getenv("LBM3D_TMA");
    const int tw = 128;
    if (!c->ref && (on && on[0] == '1') && cfg->nx % tw == 0 && (cfg->nx * (long long)c->elem) % 16 == 0 &&
        !has_halo(c)) {
      c->tma = true;
      c->tma_tw = tw;
      c->ntiles = c->g.N / tw;
      c->tma_stages = cfg->storage == LBM_STORE_FP64 ? 3 : (cfg->storage == LBM_STORE_FP16DEV ? 6 : 4);
      const char* st = std::getenv("LBM3D_TMA_STAGES");
      if (st && std::atoi(st) >= 2 && std::atoi(st) <= 8) c->tma_stages = std::atoi(st);
      if (c->cuda(cudaMalloc(&c->tiles, (size_t)c->ntiles), "cudaMalloc(tiles)")) return bail(LBM_ERR_CUDA);
      c->bytes += (size_t)c->ntiles;
    }
  }
  {
    // two cells per thread for fully periodic boxes with nx a multiple of 128: default for
    // FP32 and FP16-deviation storage (faster on B200: +2 % and +16 % on the 512^3 porous
    // box), not for FP64 (15 % slower); LBM3D_PAIR=1 / 0 forces it on / off
    const char* env = std::getenv("LBM3D_PAIR");
    const bool fits = !c->ref && !c->tma && cfg->nx % 128 == 0 && c->g.per[0] && c->g.per[1] &&
                      (c->g.per[2] || halo_only(c));
    const bool wanted = env ? env[0] == '1' : cfg->storage != LBM_STORE_FP64;
    c->pair = fits && wanted;
    // four cells per thread in the FP16-deviation even phase (aa_quad_even_kernel);
    // LBM3D_QUAD=0 keeps the pair kernels
    const char* q = std::getenv("LBM3D_QUAD");
    c->quad = c->pair && cfg->storage == LBM_STORE_FP16DEV && !(q && q[0] == '0');
    // eight cells per thread in the FP16-deviation even phase (16-byte words; nx a multiple
    // of 256; 6 % faster than four cells on the 512^3 box on B200); LBM3D_OCTO=0 keeps four
    const char* oc = std::getenv("LBM3D_OCTO");
    c->octo = c->quad && cfg->nx % 256 == 0 && !(oc && oc[0] == '0');
    // FP32 odd phase with the x-shifted directions moved as shuffled two-element words:
    // LBM3D_XSHUFFLE=1 (5 % slower than the pair kernel on the 512^3 box on B200)
    const char* xs = std::getenv("LBM3D_XSHUFFLE");
    c->xshuffle = c->pair && cfg->storage == LBM_STORE_FP32 && (xs && xs[0] == '1');
    // FP16-deviation odd phase on four cells per thread (8-byte words, x shifts exchanged
    // through shared memory; blocks of whole rows, nx at most 1024): LBM3D_QUAD_ODD=1 (22 %
    // slower than the split pair kernel on the 512^3 box on B200)
    const char* qo = std::getenv("LBM3D_QUAD_ODD");
    c->quad_odd = c->quad && cfg->nx <= 1024 && (qo && qo[0] == '1');
  }
  c->bytes += fl + ring_bytes + 64;
  if (c->cuda(cudaMemset(c->flags, 0, fl), "memset flags")) return bail(LBM_ERR_CUDA);
  if (c->cuda(cudaMemset(c->ring, 0, ring_bytes), "memset ring")) return bail(LBM_ERR_CUDA);
  if (c->A && c->cuda(cudaMemset(c->A, 0, pop), "memset populations")) return bail(LBM_ERR_CUDA);
  // the clears above run on the legacy stream, which does not order with a non-blocking
  // stream given later (lbm_set_stream): finish them before any kernel can follow
  if (c->cuda(cudaStreamSynchronize(cudaStreamLegacy), "clear")) return bail(LBM_ERR_CUDA);
  *out = c;
  return LBM_OK;
}

int32_t lbm_destroy(lbm_ctx* c) {
  if (!c) return LBM_OK;
  cudaSetDevice(c->device);
  if (c->stream) cudaStreamSynchronize(c->stream);
  cudaFree(c->A);
  for (int k = 0; k < 2; k++) {
    cudaFree(c->F[k]);
    cudaFree(c->R[k]);
  }
  cudaFree(c->flags);
  cudaFree(c->links);
  cudaFree(c->ring);
  cudaFree(c->scratch);
  cudaFree(c->d_err);
  cudaFree(c->tiles);
  delete c;
  return LBM_OK;
}

const char* lbm_last_error(const lbm_ctx* c) { return c ? c->err.c_str() : g_error.c_str(); }

int32_t lbm_set_stream(lbm_ctx* c, void* stream) {
  if (!c) return LBM_ERR_ARG;
  c->stream = (cudaStream_t)stream;
  return LBM_OK;
}

// Reads the device error word the step kernels set when a pipeline wait gives up; a
// reported failure clears the word, so the context keeps working afterwards.
static int pipeline_status(lbm_ctx* c) {
  int h = 0;
  if (c->cuda(cudaMemcpyAsync(&h, c->d_err, sizeof(int), cudaMemcpyDeviceToHost, c->stream), "D2H err")) return LBM_ERR_CUDA;
  if (c->cuda(cudaStreamSynchronize(c->stream), "cudaStreamSynchronize")) return LBM_ERR_CUDA;
  if (h) {
    if (c->cuda(cudaMemsetAsync(c->d_err, 0, sizeof(int), c->stream), "clear err")) return LBM_ERR_CUDA;
    if (c->cuda(cudaStreamSynchronize(c->stream), "cudaStreamSynchronize")) return LBM_ERR_CUDA;
    return c->fail(LBM_ERR_TIMEOUT, "a bounded mbarrier wait in a step kernel gave up (error word %d)", h);
  }
  return LBM_OK;
}

int32_t lbm_wait_selftest(lbm_ctx* c, int32_t polls) {
  if (!c) return LBM_ERR_ARG;
  if (polls < 1 || polls > MBAR_WAIT_POLLS) return c->fail(LBM_ERR_ARG, "polls %d outside [1, %d]", polls, MBAR_WAIT_POLLS);
  if (c->cuda(cudaSetDevice(c->device), "cudaSetDevice")) return LBM_ERR_CUDA;
  if (c->cuda(aa_launch_wait_probe(polls, c->d_err, c->stream), "wait probe")) return LBM_ERR_CUDA;
  return pipeline_status(c);
}

int32_t lbm_synchronize(lbm_ctx* c) {
  if (!c) return LBM_ERR_ARG;
  if (c->cuda(cudaStreamSynchronize(c->stream), "cudaStreamSynchronize")) return LBM_ERR_CUDA;
  return pipeline_status(c);
}

int64_t lbm_device_bytes(const lbm_ctx* c) { return c ? (int64_t)c->bytes : 0; }

int32_t lbm_set_launch(lbm_ctx* c, int32_t bx, int32_t by) {
  if (!c) return LBM_ERR_ARG;
  if (bx <= 0 || by <= 0 || bx * by > 256 || (bx * by) % 32 != 0)
    return c->fail(LBM_ERR_ARG, "block %dx%d: need bx*by a multiple of 32 and <= 256", bx, by);
  c->bx = bx;
  c->by = by;
  return LBM_OK;
}

int32_t lbm_get_launch(const lbm_ctx* c, int32_t* bx, int32_t* by) {
  if (!c || !bx || !by) return LBM_ERR_ARG;
  *bx = c->bx;
  *by = c->by;
  return LBM_OK;
}

int32_t lbm_add_body(lbm_ctx* c, const lbm_body* b) {
  if (!c || !b) return LBM_ERR_ARG;
  if (c->nstep > 0) return c->fail(LBM_ERR_STATE, "bodies are added before the first step");
  if (b->kind < LBM_BODY_CYLINDER_Z || b->kind > LBM_BODY_ELLIPSOID) return c->fail(LBM_ERR_ARG, "bad body kind");
  if (c->cuda(cudaSetDevice(c->device), "cudaSetDevice")) return LBM_ERR_CUDA;
  if (!c->any_body) {
    for (int a = 0; a < 3; a++) c->torque_center[a] = b->center[a];
    c->any_body = true;
  }
  if (c->cfg.solid_bc == LBM_SOLID_IBB && (!b->moving || (b->kind != LBM_BODY_CYLINDER_Z && b->kind != LBM_BODY_NACA_Z)))
    return c->fail(LBM_ERR_UNSUPPORTED, "the interpolated bounce-back takes one moving cylinder or NACA body");
  if (b->moving) {
    if (c->has_moving) return c->fail(LBM_ERR_ARG, "at most one moving body");
    if (has_halo(c)) return c->fail(LBM_ERR_UNSUPPORTED, "slabs with halo faces take static bodies only");
    c->has_moving = true;
    c->moving_body = *b;
    lbm_pose p0{};
    for (int a = 0; a < 3; a++) p0.center[a] = b->center[a];
    BodyDev d = to_dev(c, *b, nullptr);
    p0.cos_theta = d.cos_t;
    p0.sin_theta = d.sin_t;
    for (int k = 0; k < 9; k++) p0.rot[k] = b->rot[k];
    c->pose_last_step = c->pose_latest = p0;
    // rasterise both flag sets at the initial pose
    Box r = body_box(c, *b, p0.center, 2);
    if (box_clamp(c, r)) {
      FlagParams fp{};
      fp.g = c->g;
      fp.mode = c->cfg.mode;
      fp.box = r;
      fp.body = to_dev(c, *b, &p0);
      fp.body_prev = fp.body;
      fp.has_moving = 1;
      if (c->cuda(geo_launch_moving(fp, c->flags, c->stream), "moving-body flags")) return LBM_ERR_CUDA;
    }
    c->pose_bits_prev = c->pose_bits_cur = p0;
    c->kin_latest = c->kin_last_step = kin_of(p0);
  } else {
    BodyDev d = to_dev(c, *b, nullptr);
    Box r = body_box(c, *b, b->center, 2);
    if (box_clamp(c, r))
      if (c->cuda(geo_launch_static(c->g, d, r, c->flags, c->stream), "static body flags")) return LBM_ERR_CUDA;
  }
  if (near_full(c)) return LBM_ERR_CUDA;
  return c->cuda(cudaStreamSynchronize(c->stream), "add_body");
}

int32_t lbm_add_spheres(lbm_ctx* c, int32_t count, const double* xyzr) {
  if (!c || (count > 0 && !xyzr)) return LBM_ERR_ARG;
  if (c->ref) return c->fail(LBM_ERR_ARG, "lbm_add_spheres is config-mode only");
  if (c->nstep > 0) return c->fail(LBM_ERR_STATE, "bodies are added before the first step");
  if (count <= 0) return LBM_OK;
  if (c->cuda(cudaSetDevice(c->device), "cudaSetDevice")) return LBM_ERR_CUDA;
  if (!c->any_body) {
    for (int a = 0; a < 3; a++) c->torque_center[a] = xyzr[a];
    c->any_body = true;
  }
  DevBuf buf;
  const void* d = nullptr;
  if (stage_in(c, xyzr, (size_t)count * 4 * sizeof(double), LBM_HOST, buf, &d)) return LBM_ERR_CUDA;
  if (c->cuda(geo_launch_spheres(c->g, (const double*)d, count, c->flags, c->stream), "spheres")) return LBM_ERR_CUDA;
  if (near_full(c)) return LBM_ERR_CUDA;
  return c->cuda(cudaStreamSynchronize(c->stream), "add_spheres");
}

int32_t lbm_update_body(lbm_ctx* c, const lbm_pose* pn, const lbm_pose* ph) {
  if (!c || !pn) return LBM_ERR_ARG;
  const lbm_pose& half = ph ? *ph : *pn;
  c->kin_latest = kin_of(half);
  if (c->has_moving) c->pose_latest = *pn;
  return LBM_OK;
}

int32_t lbm_init_equilibrium(lbm_ctx* c, const double* rho, const double* u, const double* v, const double* w) {
  if (!c) return LBM_ERR_ARG;
  if (c->cuda(cudaSetDevice(c->device), "cudaSetDevice")) return LBM_ERR_CUDA;
  int rc = sync_flags(c);
  if (rc) return rc;
  const size_t nb = (size_t)c->g.N * sizeof(double);
  DevBuf br, bu, bv, bw;
  InitParams p{};
  p.g = c->g;
  p.rho0 = c->cfg.rho0;
  const void* dp;
  if (stage_in(c, rho, nb, LBM_HOST, br, &dp)) return LBM_ERR_CUDA;
  p.rho = (const double*)dp;
  if (stage_in(c, u, nb, LBM_HOST, bu, &dp)) return LBM_ERR_CUDA;
  p.u = (const double*)dp;
  if (stage_in(c, v, nb, LBM_HOST, bv, &dp)) return LBM_ERR_CUDA;
  p.v = (const double*)dp;
  if (stage_in(c, w, nb, LBM_HOST, bw, &dp)) return LBM_ERR_CUDA;
  p.w = (const double*)dp;
  if (c->ref) {
    for (int a = 0; a < 3; a++) p.uni[a] = 0.0;
    void* S = c->F[1 - c->ri];
    if (c->cuda(ref_launch_init(is_ref_fp64(c), p, S, c->grid(), c->block(), c->stream), "init")) return LBM_ERR_CUDA;
    RefParams rp = ref_params(c, c->kin_latest, F_SOLID);
    if (c->cuda(ref_launch_prepare(is_ref_fp64(c), c->cfg.collision == LBM_COLL_TRT, rp, S, c->F[c->ri], c->R[c->ri],
                                   c->grid(), c->block(), c->stream),
                "prepare"))
      return LBM_ERR_CUDA;
    c->ref_direct = true;
  } else {
    for (int a = 0; a < 3; a++) p.uni[a] = 0.0;
    if (c->cuda(aa_launch_init(c->cfg.storage, p, c->A, c->flags, c->grid(), c->block(), c->stream), "init"))
      return LBM_ERR_CUDA;
    c->swapped = false;
  }
  c->nstep = 0;
  c->initialised = true;
  if (c->cuda(cudaMemsetAsync(c->ring, 0, (size_t)c->ring_slots * FORCE_RECORD * sizeof(double), c->stream),
              "memset ring"))
    return LBM_ERR_CUDA;
  return c->cuda(cudaStreamSynchronize(c->stream), "init");
}

int32_t lbm_set_populations(lbm_ctx* c, const void* f, int32_t dtype, int32_t layout, int32_t where) {
  if (!c || !f) return LBM_ERR_ARG;
  if (dtype != LBM_DTYPE_F32 && dtype != LBM_DTYPE_F64) return c->fail(LBM_ERR_ARG, "bad dtype");
  if (layout != LBM_LAYOUT_SOA && layout != LBM_LAYOUT_REFERENCE) return c->fail(LBM_ERR_ARG, "bad layout");
  if (c->cuda(cudaSetDevice(c->device), "cudaSetDevice")) return LBM_ERR_CUDA;
  int rc = sync_flags(c);
  if (rc) return rc;
  DevBuf buf;
  const void* d = nullptr;
  const size_t bytes = (size_t)c->g.q * c->g.N * (dtype == LBM_DTYPE_F64 ? 8 : 4);
  if (stage_in(c, f, bytes, where, buf, &d)) return LBM_ERR_CUDA;
  InitParams p{};
  p.g = c->g;
  p.rho0 = c->cfg.rho0;
  p.f_in = d;
  p.f_dtype = dtype;
  p.f_layout = layout;
  if (c->ref) {
    void* S = c->F[1 - c->ri];
    if (c->cuda(ref_launch_init(is_ref_fp64(c), p, S, c->grid(), c->block(), c->stream), "import")) return LBM_ERR_CUDA;
    RefParams rp = ref_params(c, c->kin_latest, F_SOLID);
    if (c->cuda(ref_launch_prepare(is_ref_fp64(c), c->cfg.collision == LBM_COLL_TRT, rp, S, c->F[c->ri], c->R[c->ri],
                                   c->grid(), c->block(), c->stream),
                "prepare"))
      return LBM_ERR_CUDA;
    c->ref_direct = true;
  } else {
    if (c->cuda(aa_launch_init(c->cfg.storage, p, c->A, c->flags, c->grid(), c->block(), c->stream), "import"))
      return LBM_ERR_CUDA;
    c->swapped = false;
  }
  c->initialised = true;
  return c->cuda(cudaStreamSynchronize(c->stream), "set_populations");
}

int32_t lbm_step(lbm_ctx* c, int32_t nsteps) {
  if (!c) return LBM_ERR_ARG;
  if (!c->initialised) return c->fail(LBM_ERR_STATE, "initialise the populations first");
  if (nsteps < 0) return c->fail(LBM_ERR_ARG, "nsteps < 0");
  if (c->cuda(cudaSetDevice(c->device), "cudaSetDevice")) return LBM_ERR_CUDA;
  const bool trt = c->cfg.collision == LBM_COLL_TRT;
  for (int k = 0; k < nsteps; k++) {
    int rc = sync_flags(c);
    if (rc) return rc;
    const long long step = c->nstep + 1;  // 1-based step number being computed
    double* slot = c->ring + (size_t)(step % c->ring_slots) * FORCE_RECORD;
    double* next = c->ring + (size_t)((step + 1) % c->ring_slots) * FORCE_RECORD;
    if (c->ref) {
      RefParams p = ref_params(c, c->kin_latest, F_SOLID);
      p.compute_force = c->cfg.compute_force ? 1 : 0;
      p.force = slot;
      p.zero_next = next;
      for (int a = 0; a < 3; a++) p.kin.center[a] = c->kin_latest.center[a];
      c->launches++;
      rc = c->cuda(ref_launch_step(is_ref_fp64(c), trt, p, c->F[c->ri], c->R[c->ri], c->F[1 - c->ri], c->R[1 - c->ri],
                                   c->flags, c->grid(), c->block(), c->stream),
                   "reference step");
      if (rc) return rc;
      c->ri = 1 - c->ri;
      c->ref_direct = false;
    } else {
      AAParams p{};
      fill_aa_params(c, p, c->swapped);
      p.force = slot;
      p.zero_next = next;
      p.pair = c->pair ? 1 : 0;
      p.quad = c->pair && c->quad ? (c->swapped ? (c->quad_odd ? 1 : 0) : (c->octo ? 2 : 1)) : 0;
      p.xshuffle = c->pair && c->xshuffle ? 1 : 0;
      if (c->tma) {
        if (c->tiles_dirty) {
          c->launches++;
          rc = c->cuda(aa_launch_tile_flags(c->g, c->tma_tw, c->ntiles, c->flags, c->tiles, c->stream), "tile flags");
          if (rc) return rc;
          c->tiles_dirty = false;
        }
        TmaCfg& T = p.tma;
        T.enabled = 1;
        T.tw = c->tma_tw;
        T.halo = (int)(16 / c->elem);
        T.ntx = c->g.nx / c->tma_tw;
        T.ntiles = c->ntiles;
        T.stages = c->tma_stages;
        T.buf_elems = T.tw + T.halo;
        T.stage_bytes = (int)(((size_t)19 * T.buf_elems * c->elem + 127) / 128 * 128);
        T.tile_slow = c->tiles;
        T.err = c->d_err;
      }
      c->launches++;
      rc = c->cuda(aa_launch_step(c->cfg.storage, p, c->A, c->flags, c->swapped, trt, force_mode(c),
                                  has_faces(c) && !halo_only(c), c->grid(), c->block(), c->stream),
                   "AA step");
      if (rc) return rc;
      c->swapped = !c->swapped;
    }
    c->nstep = step;
    c->pose_last_step = c->pose_latest;
    c->kin_last_step = c->kin_latest;
  }
  return LBM_OK;
}

int64_t lbm_step_count(const lbm_ctx* c) { return c ? c->nstep : -1; }

int64_t lbm_launch_count(const lbm_ctx* c) { return c ? c->launches : -1; }

int32_t lbm_get_force_history(lbm_ctx* c, int64_t first, int32_t count, double* out) {
  if (!c || !out || count < 0) return LBM_ERR_ARG;
  if (first < 1 || first + count - 1 > c->nstep || c->nstep - first + 1 > c->cfg.force_history)
    return c->fail(LBM_ERR_ARG, "steps %lld..%lld not in the force history (last %d of %lld steps)", (long long)first,
                   (long long)(first + count - 1), c->cfg.force_history, (long long)c->nstep);
  if (c->cuda(cudaSetDevice(c->device), "cudaSetDevice")) return LBM_ERR_CUDA;
  std::vector<double> rec((size_t)count * FORCE_RECORD);
  for (int32_t k = 0; k < count; k++) {
    const long long s = first + k;
    if (c->cuda(cudaMemcpyAsync(rec.data() + (size_t)k * FORCE_RECORD, c->ring + (size_t)(s % c->ring_slots) * FORCE_RECORD,
                                FORCE_RECORD * sizeof(double), cudaMemcpyDeviceToHost, c->stream),
                "D2H force"))
      return LBM_ERR_CUDA;
  }
  if (c->cuda(cudaStreamSynchronize(c->stream), "force")) return LBM_ERR_CUDA;
  for (int32_t k = 0; k < count; k++)
    for (int j = 0; j < 6; j++) {
      double sum = 0.0;
      for (int l = 0; l < FORCE_SLOTS; l++) sum += rec[(size_t)k * FORCE_RECORD + 8 * l + j];
      out[6 * (size_t)k + j] = sum;
    }
  return LBM_OK;
}

int32_t lbm_get_force(lbm_ctx* c, int64_t step, double out[6]) { return lbm_get_force_history(c, step, 1, out); }

int32_t lbm_get_macros(lbm_ctx* c, void* rho, void* u, void* v, void* w, int32_t dtype, int32_t where) {
  if (!c) return LBM_ERR_ARG;
  if (!c->initialised) return c->fail(LBM_ERR_STATE, "not initialised");
  if (dtype != LBM_DTYPE_F32 && dtype != LBM_DTYPE_F64) return c->fail(LBM_ERR_ARG, "bad dtype");
  if (c->cuda(cudaSetDevice(c->device), "cudaSetDevice")) return LBM_ERR_CUDA;
  const size_t es = dtype == LBM_DTYPE_F64 ? 8 : 4;
  const size_t nb = (size_t)c->g.N * es;
  void* host[4] = {rho, u, v, w};
  DevBuf tmp[4];
  ExportOut out{};
  out.m_dtype = dtype;
  void* dev[4] = {nullptr, nullptr, nullptr, nullptr};
  for (int k = 0; k < 4; k++) {
    if (!host[k]) continue;
    if (where == LBM_DEVICE) {
      dev[k] = host[k];
    } else {
      if (c->cuda(cudaMalloc(&tmp[k].p, nb), "cudaMalloc(staging)")) return LBM_ERR_CUDA;
      dev[k] = tmp[k].p;
    }
  }
  out.rho = dev[0];
  out.u = dev[1];
  out.v = dev[2];
  out.w = dev[3];
  int rc;
  if (c->ref)
    rc = c->cuda(ref_launch_macros(is_ref_fp64(c), c->g, c->R[c->ri], out, c->grid(), c->block(), c->stream), "macros");
  else
    rc = export_state(c, out);
  if (rc) return rc;
  if (where == LBM_HOST) {
    for (int k = 0; k < 4; k++)
      if (host[k] && c->cuda(cudaMemcpyAsync(host[k], dev[k], nb, cudaMemcpyDeviceToHost, c->stream), "D2H macros"))
        return LBM_ERR_CUDA;
    return c->cuda(cudaStreamSynchronize(c->stream), "macros");
  }
  return LBM_OK;
}

int32_t lbm_get_populations(lbm_ctx* c, void* f, int32_t dtype, int32_t layout, int32_t where) {
  if (!c || !f) return LBM_ERR_ARG;
  if (!c->initialised) return c->fail(LBM_ERR_STATE, "not initialised");
  if (dtype != LBM_DTYPE_F32 && dtype != LBM_DTYPE_F64) return c->fail(LBM_ERR_ARG, "bad dtype");
  if (layout != LBM_LAYOUT_SOA && layout != LBM_LAYOUT_REFERENCE) return c->fail(LBM_ERR_ARG, "bad layout");
  if (c->cuda(cudaSetDevice(c->device), "cudaSetDevice")) return LBM_ERR_CUDA;
  const size_t nb = (size_t)c->g.q * c->g.N * (dtype == LBM_DTYPE_F64 ? 8 : 4);
  DevBuf tmp;
  void* dst = f;
  if (where != LBM_DEVICE) {
    if (c->cuda(cudaMalloc(&tmp.p, nb), "cudaMalloc(staging)")) return LBM_ERR_CUDA;
    dst = tmp.p;
  }
  ExportOut out{};
  out.f = dst;
  out.f_dtype = dtype;
  out.f_layout = layout;
  int rc = export_state(c, out);
  if (rc) return rc;
  if (where != LBM_DEVICE) {
    if (c->cuda(cudaMemcpyAsync(f, dst, nb, cudaMemcpyDeviceToHost, c->stream), "D2H populations")) return LBM_ERR_CUDA;
    return c->cuda(cudaStreamSynchronize(c->stream), "populations");
  }
  return LBM_OK;
}

int32_t lbm_get_flags(lbm_ctx* c, uint8_t* ms, uint8_t* mb) {
  if (!c) return LBM_ERR_ARG;
  if (c->cuda(cudaSetDevice(c->device), "cudaSetDevice")) return LBM_ERR_CUDA;
  int rc = sync_flags(c);
  if (rc) return rc;
  DevBuf a, b;
  const size_t nb = (size_t)c->g.N;
  if (ms && c->cuda(cudaMalloc(&a.p, nb), "cudaMalloc")) return LBM_ERR_CUDA;
  if (mb && c->cuda(cudaMalloc(&b.p, nb), "cudaMalloc")) return LBM_ERR_CUDA;
  if (c->cuda(geo_masks(c->g, c->cfg.mode, c->flags, F_SOLID, (uint8_t*)a.p, (uint8_t*)b.p, c->stream), "masks"))
    return LBM_ERR_CUDA;
  if (ms && c->cuda(cudaMemcpyAsync(ms, a.p, nb, cudaMemcpyDeviceToHost, c->stream), "D2H")) return LBM_ERR_CUDA;
  if (mb && c->cuda(cudaMemcpyAsync(mb, b.p, nb, cudaMemcpyDeviceToHost, c->stream), "D2H")) return LBM_ERR_CUDA;
  return c->cuda(cudaStreamSynchronize(c->stream), "flags");
}

int32_t lbm_get_links(lbm_ctx* c, int32_t* bb_ptr, int32_t* bb_lidxs, int8_t* bb_dirs, int64_t cap, int64_t* nnz) {
  if (!c || !nnz) return LBM_ERR_ARG;
  if (c->cuda(cudaSetDevice(c->device), "cudaSetDevice")) return LBM_ERR_CUDA;
  int rc = sync_flags(c);
  if (rc) return rc;
  const long long N = c->g.N;
  const long long nblk = (N + 1023) / 1024;
  DevBuf count, scan, bs, ptr, lidx, dirs;
  if (c->cuda(cudaMalloc(&count.p, (size_t)N * 4), "cudaMalloc")) return LBM_ERR_CUDA;
  if (c->cuda(cudaMalloc(&scan.p, (size_t)N * 8), "cudaMalloc")) return LBM_ERR_CUDA;
  if (c->cuda(cudaMalloc(&bs.p, (size_t)(nblk + 1) * 8), "cudaMalloc")) return LBM_ERR_CUDA;
  if (c->cuda(cudaMalloc(&ptr.p, (size_t)(N + 1) * 4), "cudaMalloc")) return LBM_ERR_CUDA;
  const long long ccap = std::max<long long>(cap, 0);
  if (ccap > 0) {
    if (c->cuda(cudaMalloc(&lidx.p, (size_t)ccap * 4), "cudaMalloc")) return LBM_ERR_CUDA;
    if (c->cuda(cudaMalloc(&dirs.p, (size_t)ccap), "cudaMalloc")) return LBM_ERR_CUDA;
  }
  long long total = 0;
  if (c->cuda(geo_links(c->g, c->cfg.mode, c->flags, F_SOLID, (int32_t*)count.p, (long long*)scan.p, (long long*)bs.p,
                        (int32_t*)ptr.p, (int32_t*)lidx.p, (int8_t*)dirs.p, ccap, &total, c->stream),
              "links"))
    return LBM_ERR_CUDA;
  *nnz = total;
  if (total >= (1LL << 31) - 1) return c->fail(LBM_ERR_CAPACITY, "more than 2^31-2 links do not fit the Int32 CSR");
  if (bb_ptr && c->cuda(cudaMemcpyAsync(bb_ptr, ptr.p, (size_t)(N + 1) * 4, cudaMemcpyDeviceToHost, c->stream), "D2H"))
    return LBM_ERR_CUDA;
  if (total <= ccap && total > 0) {
    if (bb_lidxs && c->cuda(cudaMemcpyAsync(bb_lidxs, lidx.p, (size_t)total * 4, cudaMemcpyDeviceToHost, c->stream), "D2H"))
      return LBM_ERR_CUDA;
    if (bb_dirs && c->cuda(cudaMemcpyAsync(bb_dirs, dirs.p, (size_t)total, cudaMemcpyDeviceToHost, c->stream), "D2H"))
      return LBM_ERR_CUDA;
  }
  if (c->cuda(cudaStreamSynchronize(c->stream), "links")) return LBM_ERR_CUDA;
  if (total > ccap) return c->fail(LBM_ERR_CAPACITY, "link capacity %lld < nnz %lld", ccap, total);
  return LBM_OK;
}

int32_t lbm_get_links_noalloc(lbm_ctx* c, int32_t* d_bb_ptr, int32_t* d_bb_lidxs, int8_t* d_bb_dirs, int64_t cap,
                              int64_t* nnz) {
  if (!c || !nnz || !d_bb_ptr) return LBM_ERR_ARG;
  if (cap > 0 && (!d_bb_lidxs || !d_bb_dirs)) return c->fail(LBM_ERR_ARG, "null link arrays with cap > 0");
  if (c->cuda(cudaSetDevice(c->device), "cudaSetDevice")) return LBM_ERR_CUDA;
  // the kernels write the arrays directly: each must be device (or managed) memory that
  // this context's device can address, else the call fails here instead of faulting
  {
    const void* arrs[3] = {d_bb_ptr, cap > 0 ? d_bb_lidxs : nullptr, cap > 0 ? d_bb_dirs : nullptr};
    const char* names[3] = {"d_bb_ptr", "d_bb_lidxs", "d_bb_dirs"};
    for (int k = 0; k < 3; k++) {
      if (!arrs[k]) continue;
      cudaPointerAttributes at{};
      if (cudaPointerGetAttributes(&at, arrs[k]) != cudaSuccess) {
        cudaGetLastError();  // clear the sticky-free error of an unknown pointer
        return c->fail(LBM_ERR_ARG, "%s is not a CUDA pointer", names[k]);
      }
      if (at.type != cudaMemoryTypeDevice && at.type != cudaMemoryTypeManaged)
        return c->fail(LBM_ERR_ARG, "%s is not device memory (pointer type %d)", names[k], (int)at.type);
      if (at.type == cudaMemoryTypeDevice && at.device != c->device)
        return c->fail(LBM_ERR_ARG, "%s lives on device %d, the context on device %d", names[k], at.device, c->device);
    }
  }
  if (c->g.N > geo_links_noalloc_max_nodes())
    return c->fail(LBM_ERR_CAPACITY, "lbm_get_links_noalloc supports at most %lld nodes (lattice has %lld)",
                   geo_links_noalloc_max_nodes(), c->g.N);
  int rc = sync_flags(c);
  if (rc) return rc;
  long long total = 0;
  int too_large = 0;
  if (c->cuda(geo_links_noalloc(c->g, c->cfg.mode, c->flags, F_SOLID, d_bb_ptr, d_bb_lidxs, d_bb_dirs,
                                std::max<long long>(cap, 0), &total, &too_large, c->stream),
              "links (no allocation)"))
    return LBM_ERR_CUDA;
  if (too_large)
    return c->fail(LBM_ERR_CAPACITY, "lbm_get_links_noalloc supports at most %lld nodes", geo_links_noalloc_max_nodes());
  *nnz = total;
  if (total >= (1LL << 31) - 1) return c->fail(LBM_ERR_CAPACITY, "more than 2^31-2 links do not fit the Int32 CSR");
  if (total > cap) return c->fail(LBM_ERR_CAPACITY, "link capacity %lld < nnz %lld", (long long)cap, total);
  return LBM_OK;
}

int32_t lbm_mass(lbm_ctx* c, double* out) {
  if (!c || !out) return LBM_ERR_ARG;
  if (!c->initialised) return c->fail(LBM_ERR_STATE, "not initialised");
  if (c->cuda(cudaSetDevice(c->device), "cudaSetDevice")) return LBM_ERR_CUDA;
  double r[2];
  int rc = reduce_state(c, r);
  if (rc) return rc;
  *out = r[0];
  return LBM_OK;
}

int32_t lbm_check(lbm_ctx* c) {
  if (!c) return LBM_ERR_ARG;
  if (!c->initialised) return c->fail(LBM_ERR_STATE, "not initialised");
  if (c->cuda(cudaSetDevice(c->device), "cudaSetDevice")) return LBM_ERR_CUDA;
  double r[2];
  int rc = reduce_state(c, r);
  if (rc) return rc;
  if (r[1] != 0.0) return c->fail(LBM_ERR_NUMERIC, "%.0f nodes hold non-finite populations", r[1]);
  return pipeline_status(c);
}

}  // extern "C"

// ---- batched sweeps -------------------------------------------------------------------
struct lbm_batch {
  std::vector<lbm_ctx*> ctxs;
  std::vector<BatchDom> host;  // table as last uploaded
  int device = 0;
  int storage = 0;
  bool trt = false, force = false, faces = false;
  cudaStream_t stream = nullptr;      // the members' stream
  cudaStream_t cap_stream = nullptr;  // private stream for graph capture
  BatchDom* d_doms = nullptr;
  int* d_item_dom = nullptr;
  long long* d_counter = nullptr;
  long long items = 0;
  long long k_host = 0;  // batch steps enqueued so far (= device counter once they ran)
  int blocks = 0;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  int graph_steps = 0;
  long long launches = 0;
  std::string err;

  int fail(int code, const char* fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    err = buf;
    return code;
  }
  int cuda(cudaError_t e, const char* what) {
    if (e == cudaSuccess) return LBM_OK;
    return fail(LBM_ERR_CUDA, "%s: %s", what, cudaGetErrorString(e));
  }
};

namespace {

// Table entry of member m for batch step k_host: the domain has completed
// ctx->nstep steps and its populations are in the `swapped` layout.
void batch_entry(const lbm_batch* b, int m, BatchDom& e) {
  const lbm_ctx* c = b->ctxs[m];
  const long long item_begin = e.item_begin, item_end = e.item_end;
  e = BatchDom{};
  fill_aa_params(c, e.p[0], false);
  fill_aa_params(c, e.p[1], true);
  e.A = c->A;
  e.flags = c->flags;
  e.ring = c->ring;
  e.ring_slots = c->ring_slots;
  e.base_step = c->nstep - b->k_host;
  e.phase0 = (int)(((c->swapped ? 1 : 0) - (b->k_host & 1) + 2) & 1);
  e.item_begin = item_begin;
  e.item_end = item_end;
}

// Brings the device table in line with the members (a member stepped alone since the
// last batch call) and orders the batch after work on the members' stream.
int batch_refresh(lbm_batch* b) {
  bool dirty = false;
  for (size_t m = 0; m < b->ctxs.size(); m++) {
    const lbm_ctx* c = b->ctxs[m];
    const BatchDom& e = b->host[m];
    const bool swapped = ((e.phase0 + b->k_host) & 1) != 0;
    if (e.base_step + b->k_host != c->nstep || swapped != c->swapped) {
      batch_entry(b, (int)m, b->host[m]);
      dirty = true;
    }
  }
  if (dirty &&
      b->cuda(cudaMemcpyAsync(b->d_doms, b->host.data(), b->host.size() * sizeof(BatchDom), cudaMemcpyHostToDevice,
                              b->stream),
              "upload batch table"))
    return LBM_ERR_CUDA;
  // pageable source: the copy is staged before cudaMemcpyAsync returns
  return LBM_OK;
}

void batch_advance_members(lbm_batch* b, long long n) {
  b->k_host += n;
  for (lbm_ctx* c : b->ctxs) {
    c->nstep += n;
    if (n & 1) c->swapped = !c->swapped;
    c->pose_last_step = c->pose_latest;
    c->kin_last_step = c->kin_latest;
  }
}

int batch_enqueue(lbm_batch* b, int nsteps, cudaStream_t s) {
  BatchParams bp{};
  bp.doms = b->d_doms;
  bp.item_dom = b->d_item_dom;
  bp.items = b->items;
  bp.counter = b->d_counter;
  for (int k = 0; k < nsteps; k++) {
    if (b->cuda(aa_launch_batch(b->storage, bp, b->trt, b->force, b->faces, b->blocks, s), "batched step"))
      return LBM_ERR_CUDA;
    if (b->cuda(aa_launch_batch_advance(b->d_counter, s), "batch counter")) return LBM_ERR_CUDA;
  }
  return LBM_OK;
}

void batch_free(lbm_batch* b) {
  if (b->exec) cudaGraphExecDestroy(b->exec);
  if (b->graph) cudaGraphDestroy(b->graph);
  if (b->cap_stream) cudaStreamDestroy(b->cap_stream);
  cudaFree(b->d_doms);
  cudaFree(b->d_item_dom);
  cudaFree(b->d_counter);
}

}  // namespace

extern "C" {

int32_t lbm_batch_create(lbm_ctx* const* ctxs, int32_t count, lbm_batch** out) {
  if (!ctxs || !out || count < 1) return set_global(LBM_ERR_ARG, "lbm_batch_create: need at least one context");
  *out = nullptr;
  const lbm_ctx* c0 = ctxs[0];
  if (!c0) return set_global(LBM_ERR_ARG, "lbm_batch_create: null context 0");
  long long items = 0;
  for (int32_t m = 0; m < count; m++) {
    const lbm_ctx* c = ctxs[m];
    if (!c) return set_global(LBM_ERR_ARG, "lbm_batch_create: null context %d", m);
    if (c->ref) return set_global(LBM_ERR_UNSUPPORTED, "context %d: batches take config-mode domains", m);
    if (!c->initialised) return set_global(LBM_ERR_STATE, "context %d is not initialised", m);
    if (c->has_moving) return set_global(LBM_ERR_UNSUPPORTED, "context %d has a moving body (batches take static bodies)", m);
    if (c->tma) return set_global(LBM_ERR_UNSUPPORTED, "context %d uses the TMA-staged step", m);
    if (c->device != c0->device || c->stream != c0->stream)
      return set_global(LBM_ERR_ARG, "context %d: all members share one device and one stream", m);
    if (c->cfg.storage != c0->cfg.storage || c->cfg.collision != c0->cfg.collision)
      return set_global(LBM_ERR_ARG, "context %d: all members share storage and collision", m);
    for (int32_t j = 0; j < m; j++)
      if (ctxs[j] == c) return set_global(LBM_ERR_ARG, "context %d appears twice", m);
    items += (c->g.N + BATCH_ITEM - 1) / BATCH_ITEM;
  }
  if (items >= (1LL << 31)) return set_global(LBM_ERR_CAPACITY, "more than 2^31-1 work items");
  lbm_batch* b = new lbm_batch();
  b->ctxs.assign(ctxs, ctxs + count);
  b->device = c0->device;
  b->stream = c0->stream;
  b->storage = c0->cfg.storage;
  b->trt = c0->cfg.collision == LBM_COLL_TRT;
  b->items = items;
  for (lbm_ctx* c : b->ctxs) {
    b->force = b->force || has_force(c);  // a zero acceleration adds exact zeros
    b->faces = b->faces || has_faces(c);
  }
  auto bail = [&](int rc) {
    set_global(rc, "%s", b->err.c_str());
    batch_free(b);
    delete b;
    return rc;
  };
  if (b->cuda(cudaSetDevice(b->device), "cudaSetDevice")) return bail(LBM_ERR_CUDA);
  b->host.resize(count);
  std::vector<int> item_dom((size_t)items);
  long long next = 0;
  for (int32_t m = 0; m < count; m++) {
    const long long n = (ctxs[m]->g.N + BATCH_ITEM - 1) / BATCH_ITEM;
    b->host[m].item_begin = next;
    b->host[m].item_end = next + n;
    for (long long i = 0; i < n; i++) item_dom[(size_t)(next + i)] = m;
    next += n;
    batch_entry(b, m, b->host[m]);
  }
  int per_sm = 0, sms = 0;
  if (b->cuda(aa_batch_blocks_per_sm(b->storage, b->trt, b->force, b->faces, &per_sm), "occupancy")) return bail(LBM_ERR_CUDA);
  if (b->cuda(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, b->device), "SM count")) return bail(LBM_ERR_CUDA);
  if (per_sm < 1) return bail(b->fail(LBM_ERR_CUDA, "the batched kernel does not fit on an SM"));
  b->blocks = (int)std::min<long long>((long long)sms * per_sm, items);
  if (const char* env = std::getenv("LBM3D_BATCH_BLOCKS")) {
    const int v = std::atoi(env);
    if (v > 0) b->blocks = (int)std::min<long long>(v, items);
  }
  if (b->cuda(cudaMalloc(&b->d_doms, (size_t)count * sizeof(BatchDom)), "cudaMalloc(batch table)")) return bail(LBM_ERR_CUDA);
  if (b->cuda(cudaMalloc(&b->d_item_dom, (size_t)items * sizeof(int)), "cudaMalloc(item map)")) return bail(LBM_ERR_CUDA);
  if (b->cuda(cudaMalloc(&b->d_counter, sizeof(long long)), "cudaMalloc(counter)")) return bail(LBM_ERR_CUDA);
  // on the members' stream (it may be non-blocking, so legacy-stream copies would not
  // order with the batch's kernels); the synchronisation below also ends the members'
  // earlier work (initialisation, single steps) before the batch
  if (b->cuda(cudaMemcpyAsync(b->d_doms, b->host.data(), (size_t)count * sizeof(BatchDom), cudaMemcpyHostToDevice,
                              b->stream),
              "H2D"))
    return bail(LBM_ERR_CUDA);
  if (b->cuda(cudaMemcpyAsync(b->d_item_dom, item_dom.data(), (size_t)items * sizeof(int), cudaMemcpyHostToDevice,
                              b->stream),
              "H2D"))
    return bail(LBM_ERR_CUDA);
  if (b->cuda(cudaMemsetAsync(b->d_counter, 0, sizeof(long long), b->stream), "memset")) return bail(LBM_ERR_CUDA);
  if (b->cuda(cudaStreamSynchronize(b->stream), "cudaStreamSynchronize")) return bail(LBM_ERR_CUDA);
  *out = b;
  return LBM_OK;
}

int32_t lbm_batch_destroy(lbm_batch* b) {
  if (!b) return LBM_OK;
  cudaSetDevice(b->device);
  cudaStreamSynchronize(b->stream);
  batch_free(b);
  delete b;
  return LBM_OK;
}

const char* lbm_batch_last_error(const lbm_batch* b) { return b ? b->err.c_str() : g_error.c_str(); }

int32_t lbm_batch_step(lbm_batch* b, int32_t nsteps) {
  if (!b) return LBM_ERR_ARG;
  if (nsteps < 0) return b->fail(LBM_ERR_ARG, "nsteps < 0");
  if (b->cuda(cudaSetDevice(b->device), "cudaSetDevice")) return LBM_ERR_CUDA;
  int rc = batch_refresh(b);
  if (rc) return rc;
  rc = batch_enqueue(b, nsteps, b->stream);
  if (rc) return rc;
  b->launches += (long long)BATCH_LAUNCHES_PER_STEP * nsteps;
  for (lbm_ctx* c : b->ctxs) c->launches += nsteps;
  batch_advance_members(b, nsteps);
  return LBM_OK;
}

int32_t lbm_batch_capture(lbm_batch* b, int32_t nsteps) {
  if (!b) return LBM_ERR_ARG;
  if (nsteps < 1) return b->fail(LBM_ERR_ARG, "nsteps < 1");
  if (b->cuda(cudaSetDevice(b->device), "cudaSetDevice")) return LBM_ERR_CUDA;
  if (b->exec) {
    cudaGraphExecDestroy(b->exec);
    b->exec = nullptr;
  }
  if (b->graph) {
    cudaGraphDestroy(b->graph);
    b->graph = nullptr;
  }
  if (!b->cap_stream &&
      b->cuda(cudaStreamCreateWithFlags(&b->cap_stream, cudaStreamNonBlocking), "cudaStreamCreate"))
    return LBM_ERR_CUDA;
  if (b->cuda(cudaStreamBeginCapture(b->cap_stream, cudaStreamCaptureModeThreadLocal), "begin capture"))
    return LBM_ERR_CUDA;
  const int rc = batch_enqueue(b, nsteps, b->cap_stream);
  cudaGraph_t g = nullptr;
  const cudaError_t e = cudaStreamEndCapture(b->cap_stream, &g);
  if (rc) {
    if (g) cudaGraphDestroy(g);
    return rc;
  }
  if (b->cuda(e, "end capture")) return LBM_ERR_CUDA;
  b->graph = g;
  if (b->cuda(cudaGraphInstantiate(&b->exec, b->graph, 0), "cudaGraphInstantiate")) return LBM_ERR_CUDA;
  b->graph_steps = nsteps;
  return LBM_OK;
}

int32_t lbm_batch_replay(lbm_batch* b, int32_t times) {
  if (!b) return LBM_ERR_ARG;
  if (!b->exec) return b->fail(LBM_ERR_STATE, "no captured graph (call lbm_batch_capture first)");
  if (times < 0) return b->fail(LBM_ERR_ARG, "times < 0");
  if (b->cuda(cudaSetDevice(b->device), "cudaSetDevice")) return LBM_ERR_CUDA;
  int rc = batch_refresh(b);
  if (rc) return rc;
  for (int32_t r = 0; r < times; r++)
    if (b->cuda(cudaGraphLaunch(b->exec, b->stream), "cudaGraphLaunch")) return LBM_ERR_CUDA;
  const long long n = (long long)times * b->graph_steps;
  b->launches += (long long)BATCH_LAUNCHES_PER_STEP * n;
  for (lbm_ctx* c : b->ctxs) c->launches += n;
  batch_advance_members(b, n);
  return LBM_OK;
}

int64_t lbm_batch_launch_count(const lbm_batch* b) { return b ? b->launches : -1; }

int32_t lbm_batch_synchronize(lbm_batch* b) {
  if (!b) return LBM_ERR_ARG;
  if (b->cuda(cudaSetDevice(b->device), "cudaSetDevice")) return LBM_ERR_CUDA;
  return b->cuda(cudaStreamSynchronize(b->stream), "cudaStreamSynchronize");
}

// ---- z-slab halo messages ----
int64_t lbm_halo_bytes(const lbm_ctx* c) {
  if (!c || !has_halo(c)) return 0;
  return 5LL * c->g.nx * c->g.ny * c->elem;
}

static int32_t halo_call(lbm_ctx* c, int32_t side, const void* buf, bool pack) {
  if (!c || !buf) return LBM_ERR_ARG;
  if (side != 0 && side != 1) return c->fail(LBM_ERR_ARG, "side must be 0 (z-lo) or 1 (z-hi)");
  if (c->ref || c->cfg.face[4 + side] != LBM_FACE_HALO)
    return c->fail(LBM_ERR_ARG, "face %d is not a halo face", 4 + side);
  if (!c->initialised) return c->fail(LBM_ERR_STATE, "initialise the populations first");
  if (c->cuda(cudaSetDevice(c->device), "cudaSetDevice")) return LBM_ERR_CUDA;
  // swapped layout <=> the last step was an even-phase step
  return c->cuda(aa_launch_halo(c->g, c->elem, side, c->swapped, pack, c->A, c->flags, const_cast<void*>(buf),
                                c->stream),
                 pack ? "halo pack" : "halo unpack");
}

int32_t lbm_halo_pack(lbm_ctx* c, int32_t side, void* d_buf) { return halo_call(c, side, d_buf, true); }
int32_t lbm_halo_unpack(lbm_ctx* c, int32_t side, const void* d_buf) { return halo_call(c, side, d_buf, false); }

}  // extern "C"
