"""Table-driven numpy transliteration of the reference step (one partition).

TEST INFRASTRUCTURE ONLY — a second, independent restatement used to check the C++
oracle.  Where lbm_oracle.cpp computes neighbours by index arithmetic, this module
builds the reference's own lookup tables and applies the kernels one after another
on two population arrays, in float32 with the reference's operation order:

  lattice            gen_lattice_sets            Utilities.jl:945-993
  node tables        build_local_tables          Utilities.jl:520-575  (x_lli, nbr_lli)
  stream table       build_stream_lists          Utilities.jl:734-790  (+ per_mask)
  face lists         compile_face_BC             Utilities.jl:795-855
  periodic lists     compile_periodic_BC         Utilities.jl:860-898
  solid mask         generate_mask_s_local!_gpu  Geometry.jl:49-87 (cylinder)
  boundary mask      generate_mask_bb_local!_gpu Geometry.jl:122-148
  link CSR           compile_bb_data!            Geometry.jl:181-311
  collision          BGK/TRT_collision!_gpu      Collision.jl:112-174, 212-242
  streaming          streaming!_gpu              Streaming.jl:82-111
  periodic copy      periodic_BC!_gpu            OtherBC.jl:65-82
  solid BC           SBB!_gpu                    SolidBC.jl:160-210
  face BCs           velocity_BC!_gpu            OtherBC.jl:112-169 (pressure entries after velocity)
  momentum exchange  momentum_exchange_gpu       MEA.jl:76-116 (FP64 sum here)
  macros             compute_macros!_gpu         ComputeMacro.jl:11-48

Indices follow the reference (1-based node and direction numbers in the tables),
converted to 0-based only when indexing numpy arrays.  Slow (pure Python loops over
the tables); intended for domains of a few thousand nodes.
"""
from __future__ import annotations

import numpy as np

F = np.float32

CX = [1, -1, 0, 0, 0, 0, 1, -1, 1, -1, 0, 0, 1, -1, 1, -1, 0, 0, 0]
CY = [0, 0, 1, -1, 0, 0, 1, -1, 0, 0, 1, -1, -1, 1, 0, 0, 1, -1, 0]
CZ = [0, 0, 0, 0, 1, -1, 0, 0, 1, -1, 1, -1, 0, 0, -1, 1, -1, 1, 0]
BBOPP = [2, 1, 4, 3, 6, 5, 8, 7, 10, 9, 12, 11, 14, 13, 16, 15, 18, 17, 19]
W = [F(1) / F(18)] * 6 + [F(1) / F(36)] * 12 + [F(1) / F(3)]
Q = 19


class TableReference:
    def __init__(self, Nx, Ny, Nz, *, h, omega_p, omega_m, coll, U_inf, V_inf=0.0, W_inf=0.0, R=None):
        self.Nx, self.Ny, self.Nz = Nx, Ny, Nz
        self.h = F(h)
        self.omega_p, self.omega_m = F(omega_p), F(omega_m)
        self.coll = coll
        self.U, self.V, self.Wz = F(U_inf), F(V_inf), F(W_inf)
        self.R = F(R) if R is not None else None
        N = Nx * Ny * Nz
        self.N = N
        # global order (Partitioning.jl:23-28): g = (iz-1)NxNy + (iy-1)Nx + ix
        self.xyz = [None] * (N + 1)
        g = 1
        for iz in range(1, Nz + 1):
            for iy in range(1, Ny + 1):
                for ix in range(1, Nx + 1):
                    self.xyz[g] = (ix, iy, iz)
                    g += 1
        self._tables()
        self.f_old = np.zeros((N, Q), F)  # f[node, d] == reference f[d, node]
        self.f_new = np.zeros((N, Q), F)
        self.rho = np.zeros(N, F)
        self.u = np.zeros(N, F)
        self.v = np.zeros(N, F)
        self.w = np.zeros(N, F)

    def gidx(self, ix, iy, iz):
        return (iz - 1) * self.Nx * self.Ny + (iy - 1) * self.Nx + ix

    # ---- tables --------------------------------------------------------------------
    def _tables(self):
        Nx, Ny, Nz, N = self.Nx, self.Ny, self.Nz, self.N
        # build_local_tables: x_lli, y_lli, nbr_lli (-1 off the domain)
        self.x_lli = np.zeros(N + 1, F)
        self.y_lli = np.zeros(N + 1, F)
        self.nbr = np.full((N + 1, Q), -1, np.int64)
        for a in range(1, N + 1):
            ix, iy, iz = self.xyz[a]
            self.x_lli[a] = (F(ix) - F(0.5)) * self.h
            self.y_lli[a] = (F(iy) - F(0.5)) * self.h
            for q in range(Q):
                jx, jy, jz = ix + CX[q], iy + CY[q], iz + CZ[q]
                if 1 <= jx <= Nx and 1 <= jy <= Ny and 1 <= jz <= Nz:
                    self.nbr[a, q] = self.gidx(jx, jy, jz)
        # build_stream_lists + per_mask
        self.stream = np.zeros((N + 1, Q), np.int64)
        self.per_mask = np.zeros((N + 1, Q), np.uint8)
        for i in range(1, N + 1):
            gx, gy, gz = self.xyz[i]
            for d in range(Q):
                nx, ny, nz = gx - CX[d], gy - CY[d], gz - CZ[d]
                if 1 <= nx <= Nx and 1 <= ny <= Ny and 1 <= nz <= Nz:
                    src = self.gidx(nx, ny, nz)
                else:
                    src = i
                    if (nz < 1 or nz > Nz) and 1 <= nx <= Nx and 1 <= ny <= Ny:
                        self.per_mask[i, d] = 1
                self.stream[i, d] = src
        # compile_face_BC
        self.vel, self.pres = [], []
        for i in range(1, N + 1):
            x, y, z = self.xyz[i]
            if x == 1:
                self.vel += [(i, d + 1) for d in range(Q) if CX[d] > 0]
            if y == 1:
                self.vel += [(i, d + 1) for d in range(Q) if CY[d] > 0]
            if y == Ny:
                self.vel += [(i, d + 1) for d in range(Q) if CY[d] < 0]
            if x == Nx:
                self.pres += [(i, d + 1) for d in range(Q) if CX[d] < 0]
        # compile_periodic_BC
        self.per = []
        for i in range(1, N + 1):
            x, y, z = self.xyz[i]
            for d in range(Q):
                dx, dy, dz = CX[d], CY[d], CZ[d]
                if z + dz < 1 or z + dz > Nz:
                    zs = ((z + dz - 1) % Nz) + 1
                    xs, ys = x + dx, y + dy
                    if 1 <= xs <= Nx and 1 <= ys <= Ny:
                        self.per.append((i, self.gidx(xs, ys, zs), BBOPP[d]))

    # ---- geometry --------------------------------------------------------------------
    def masks(self, x_c, y_c):
        """generate_mask_s_local! (cylinder) and generate_mask_bb_local!."""
        N = self.N
        R2 = self.R * self.R
        ms = np.zeros(N + 1, bool)
        for a in range(1, N + 1):
            dx = self.x_lli[a] - F(x_c)
            dy = self.y_lli[a] - F(y_c)
            ms[a] = (dx * dx + dy * dy) <= (R2 + F(1e-6) * R2)
        mb = np.zeros(N + 1, bool)
        for a in range(1, N + 1):
            if ms[a]:
                continue
            for q in range(Q):
                b = self.nbr[a, q]
                if b != -1 and ms[b]:
                    mb[a] = True
                    break
        return ms, mb

    def links(self, ms, mb):
        """compile_bb_data!: count, inclusive scan, ptr, fill (1-based CSR)."""
        N = self.N
        cnt = np.zeros(N + 1, np.int64)
        for a in range(1, N + 1):
            if mb[a]:
                cnt[a] = sum(1 for q in range(Q) if self.nbr[a, q] != -1 and ms[self.nbr[a, q]])
        scan = np.cumsum(cnt[1:])
        ptr = np.zeros(N + 1, np.int64)
        ptr[0] = 1
        ptr[1:] = 1 + scan
        dirs, lidx = [], []
        for a in range(1, N + 1):
            if ptr[a] == ptr[a - 1]:
                continue
            for q in range(Q):
                b = self.nbr[a, q]
                if b != -1 and ms[b]:
                    dirs.append(q + 1)
                    lidx.append(a)
        return ptr.astype(np.int32), np.array(lidx, np.int32), np.array(dirs, np.int8)

    # ---- kernels -----------------------------------------------------------------------
    def init(self, rho, u, v, w):
        for i in range(self.N):
            for d in range(Q):
                cu = F(CX[d]) * F(u[i]) + F(CY[d]) * F(v[i]) + F(CZ[d]) * F(w[i])
                u2 = F(u[i]) * F(u[i]) + F(v[i]) * F(v[i]) + F(w[i]) * F(w[i])
                cu2 = cu * cu
                self.f_old[i, d] = W[d] * F(rho[i]) * (F(1) + cu * F(3) + F(0.5) * cu2 * F(9) - F(0.5) * u2 * F(3))
        self.f_new[:] = self.f_old
        self.macros()

    def macros(self):
        for i in range(self.N):
            r = F(0)
            mx = my = mz = F(0)
            for d in range(Q):
                f = self.f_old[i, d]
                r = r + f
                mx = mx + f * F(CX[d])
                my = my + f * F(CY[d])
                mz = mz + f * F(CZ[d])
            self.rho[i] = r
            self.u[i] = mx / r
            self.v[i] = my / r
            self.w[i] = mz / r

    def collision(self):
        for i in range(self.N):
            r, ux, uy, uz = self.rho[i], self.u[i], self.v[i], self.w[i]
            if self.coll == "BGK":
                for d in range(Q):
                    cu = F(CX[d]) * ux + F(CY[d]) * uy + F(CZ[d]) * uz
                    cu2 = cu * cu
                    u2 = ux * ux + uy * uy + uz * uz
                    feq = W[d] * r * (F(1) + cu * F(3) + F(0.5) * cu2 * F(9) - F(0.5) * u2 * F(3))
                    fo = self.f_old[i, d]
                    self.f_new[i, d] = fo - self.omega_p * (fo - feq)
            else:
                u2 = ux * ux + uy * uy + uz * uz
                for d in range(Q):
                    q = BBOPP[d] - 1
                    fi, fo = self.f_old[i, d], self.f_old[i, q]
                    cu = F(CX[d]) * ux + F(CY[d]) * uy + F(CZ[d]) * uz
                    cu2 = cu * cu
                    fp_eq = W[d] * r * (F(1) + F(0.5) * cu2 * F(9) - F(0.5) * u2 * F(3))
                    fm_eq = W[d] * r * (cu * F(3))
                    fp = F(0.5) * (fi + fo)
                    fm = F(0.5) * (fi - fo)
                    self.f_new[i, d] = (fp - self.omega_p * (fp - fp_eq)) + (fm - self.omega_m * (fm - fm_eq))

    def streaming(self):
        for i in range(1, self.N + 1):
            for d in range(Q):
                if self.per_mask[i, d] == 1:
                    continue
                self.f_old[i - 1, d] = self.f_new[self.stream[i, d] - 1, d]

    def periodic(self):
        for dest, src, dr in self.per:
            self.f_old[dest - 1, dr - 1] = self.f_new[src - 1, dr - 1]

    def sbb(self, lidx, dirs, U, V, om, xcl, ycl):
        for i, dr in zip(lidx, dirs):
            d = dr - 1
            o = BBOPP[d] - 1
            cx, cy = F(CX[d]), F(CY[d])
            xlat = self.x_lli[i] / self.h
            ylat = self.y_lli[i] / self.h
            xw = xlat - F(0.5) * cx
            yw = ylat - F(0.5) * cy
            rx, ry = xw - F(xcl), yw - F(ycl)
            uwx = F(U) - F(om) * ry
            uwy = F(V) + F(om) * rx
            cdu = cx * uwx + cy * uwy
            self.f_old[i - 1, o] = self.f_new[i - 1, d] - F(2) * W[d] * self.rho[i - 1] * cdu * F(3)

    def velocity_bc(self):
        for i, dr in self.vel:
            d = dr - 1
            o = BBOPP[d] - 1
            cu = F(CX[d]) * (-self.U) + F(CY[d]) * (-self.V) + F(CZ[d]) * (-self.Wz)
            self.f_old[i - 1, d] = self.f_new[i - 1, o] - F(2) * W[d] * self.rho[i - 1] * cu * F(3)
        for i, dr in self.pres:
            d = dr - 1
            o = BBOPP[d] - 1
            uw, vw, ww = self.u[i - 1], self.v[i - 1], self.w[i - 1]
            cu = F(CX[d]) * uw + F(CY[d]) * vw + F(CZ[d]) * ww
            cu2 = cu * cu
            uu2 = uw * uw + vw * vw + ww * ww
            self.f_old[i - 1, d] = -self.f_new[i - 1, o] + F(2) * W[d] * self.rho[i - 1] * (
                F(1) + F(0.5) * cu2 * F(9) - F(0.5) * uu2 * F(3))

    def mea(self, lidx, dirs):
        P = np.zeros(3)
        for i, dr in zip(lidx, dirs):
            d = dr - 1
            o = BBOPP[d] - 1
            t = float(self.f_new[i - 1, d]) + float(self.f_old[i - 1, o])
            P += t * np.array([CX[d], CY[d], CZ[d]], float)
        return P

    def step(self, pose_n, kin_half):
        """One pass of MainCore.jl:245-379 (no halo exchange at one partition)."""
        ms, mb = self.masks(*pose_n)
        ptr, lidx, dirs = self.links(ms, mb)
        self.collision()
        self.streaming()
        self.periodic()
        self.sbb(lidx, dirs, *kin_half)
        self.velocity_bc()
        P = self.mea(lidx, dirs)
        self.macros()
        return P, (ms[1:], mb[1:], ptr, lidx, dirs)
