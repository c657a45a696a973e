"""FP64 numpy restatement of the ESP pipeline (test infrastructure only).

Stage-by-stage CPU restatement of the hot path, following the reference's
stage order (``src/ESPForceCompute.cc:96-127``) and layouts, with the
corrected mathematics described in ``esp_hoomd_b200.tables``:

* bin + sort: cell key of each particle's first stencil point, stable sort
  on (key, index) -- new stage; the nearest reference code is
  ``box.makeFraction`` + ``floorf`` in ``src/ESPForceComputeGPU.cu:228-236``.
* weights: one local coordinate ``t`` per axis, P polynomial segments
  (replaces ``gpu_eval_stencil_weight``, ``src/ESPForceComputeGPU.cu:138-152``).
* spread: ``rho[cell] += q wx wy wz`` over the P^3 periodic stencil, mesh
  x-fastest ``cell = (cz*ny + cy)*nx + cx`` (``src/ESPForceComputeGPU.cu:206-272``).
* forward FFT (``src/ESPForceComputeGPU.cc:254-265``), influence multiply
  (``src/ESPForceComputeGPU.cu:277-287``), inverse FFT (missing in the
  reference, ``src/ESPForceCompute.cc:225-232``).
* interpolation with analytic differentiation of the window
  (``src/ESPForceComputeGPU.cu:292-373`` gathers three ik meshes instead).
* pair term over a CSR neighbour list: ``EvaluatorPairPSWF`` semantics
  (``src/EvaluatorPairPSWF.h:274-295``) with the split polynomial.
* energies: reciprocal (1/2 sum q phi), self, neutralising background, and
  the k-space virial (stubs in the reference, ``src/ESPForceCompute.cc:236-248``).

Everything here is float64; the GPU path is checked against it.
"""
from __future__ import annotations

import math
from typing import Optional, Sequence

import numpy as np

INV_4PI = 0.079577471545947673
PSI_FLOOR = 1e-14


def wrap_f32(pos, box):
    """Positions wrapped into [0, L) in float32 (x - L floor(x / L))."""
    p = np.asarray(pos, dtype=np.float32)
    L = np.asarray(box, dtype=np.float64).astype(np.float32)
    inv = (np.float32(1.0) / L).astype(np.float32)
    x = (p - L * np.floor(p * inv)).astype(np.float32)
    x = np.where(x >= L, x - L, x)
    x = np.where(x < 0, x + L, x)
    return x.astype(np.float32)


def grid_coords(pos, box, mesh):
    """Grid coordinate g = x (n / L) per axis, x the float32 position
    wrapped into the box, the product taken in FP64 (the
    ``box.makeFraction(pos) * mesh_dim`` of ``src/ESPForceComputeGPU.cu:228-233``)."""
    x = wrap_f32(pos, box).astype(np.float64)
    L = np.asarray(box, dtype=np.float64)
    n = np.asarray(mesh, dtype=np.float64)
    g = x * (n / L)
    return np.where(g >= n, g - n, g)


def stencil_origin(g, P):
    """First stencil point i0 = floor(g - P/2) + 1 and local t = i0 + P/2 - g."""
    i0 = np.floor(g - 0.5 * P).astype(np.int64) + 1
    t = i0 + 0.5 * P - g
    return i0, t


def bin_sort(pos, box, mesh, P, tile):
    """Tile key of each particle and the stable permutation by (key, y origin
    inside the tile, index).

    key = linear tile index (x-fastest) of the tile holding the particle's
    first stencil point i0 (mod n); tiles are ``tile^3`` mesh cells. Inside a
    tile particles are ordered by the y coordinate of their first stencil
    point relative to the tile, then by index.
    Returns (key uint32[N], perm uint32[N]).
    """
    g = grid_coords(pos, box, mesh)
    i0, _ = stencil_origin(g, P)
    n = np.asarray(mesh, dtype=np.int64)
    c = np.mod(i0, n)
    nt = (n + tile - 1) // tile
    tc = c // tile
    key = ((tc[:, 2] * nt[1] + tc[:, 1]) * nt[0] + tc[:, 0]).astype(np.uint32)
    oy = c[:, 1] - tc[:, 1] * tile
    perm = np.lexsort((np.arange(key.size), oy, key)).astype(np.uint32)
    return key, perm


def influence(params, kind: str = "G"):
    """Half-spectrum influence table G[kz, ky, kx] (kx in [0, nx//2]).

    ``G = Psi(|k| r_c) / (|k|^2 V wx^2 wy^2 wz^2)`` with w the grid-unit
    Fourier transform of the fitted window, G(0)=0 (reference K1 builds
    ``exp(-k^2/4kappa^2)/(k^2 b(k^2))`` instead, ``src/ESPForceComputeGPU.cu:157-201``).
    kind="B" returns the virial factor ``B(k) = -2/k^2 + r_c Psi'(k r_c)/(k Psi)``.
    """
    nx, ny, nz = params.mesh
    Lx, Ly, Lz = params.box
    V = Lx * Ly * Lz
    kx = 2 * math.pi * np.arange(nx // 2 + 1) / Lx
    ky = 2 * math.pi * np.fft.fftfreq(ny, 1.0 / ny) / Ly
    kz = 2 * math.pi * np.fft.fftfreq(nz, 1.0 / nz) / Lz
    wx = params.window.fourier(kx * Lx / nx)
    wy = params.window.fourier(ky * Ly / ny)
    wz = params.window.fourier(kz * Lz / nz)
    KZ, KY, KX = np.meshgrid(kz, ky, kx, indexing="ij")
    k2 = KX * KX + KY * KY + KZ * KZ
    kk = np.sqrt(k2)
    rc = params.rcut
    kap = (kk * rc).ravel()
    # Psi on the distinct |k| values only
    uk, inv = np.unique(np.round(kap, 12), return_inverse=True)
    psi_u = params.split.fourier_ratio(uk)
    psi = psi_u[inv].reshape(k2.shape)
    W2 = (wz[:, None, None] * wy[None, :, None] * wx[None, None, :]) ** 2
    # modes whose Psi is below 1e-14 are dropped (their de-convolved weight
    # would only amplify aliasing noise)
    psi = np.where(psi > PSI_FLOOR, psi, 0.0)
    # Nyquist planes of even meshes are dropped (Psi there is at the split's
    # truncation level, and 1/w^2 amplifies aliasing the most)
    if nx % 2 == 0:
        psi[:, :, nx // 2] = 0.0
    if ny % 2 == 0:
        psi[:, ny // 2, :] = 0.0
    if nz % 2 == 0:
        psi[nz // 2, :, :] = 0.0
    with np.errstate(divide="ignore", invalid="ignore"):
        G = np.where(k2 > 0, psi / (k2 * V * W2), 0.0)
        if kind == "G":
            return G
        h = 1e-6
        dpsi_u = (params.split.fourier_ratio(uk + h) - params.split.fourier_ratio(np.maximum(uk - h, 0))) / \
            (uk + h - np.maximum(uk - h, 0))
        dpsi = dpsi_u[inv].reshape(k2.shape)
        B = np.where(k2 > 0, -2.0 / k2 + rc * dpsi / (kk * np.where(psi != 0, psi, 1.0)), 0.0)
        return B


def spread(pos, q, params):
    """Charge mesh rho[z, y, x] (float64)."""
    nx, ny, nz = params.mesh
    P = params.P
    g = grid_coords(pos, params.box, params.mesh)
    i0, t = stencil_origin(g, P)
    wx = params.window.weights(t[:, 0])
    wy = params.window.weights(t[:, 1])
    wz = params.window.weights(t[:, 2])
    mesh = np.zeros((nz, ny, nx))
    a = np.arange(P)
    cx = np.mod(i0[:, 0:1] + a, nx)
    cy = np.mod(i0[:, 1:2] + a, ny)
    cz = np.mod(i0[:, 2:3] + a, nz)
    for c in range(P):
        w = q[:, None, None] * wz[:, c, None, None] * wy[:, :, None] * wx[:, None, :]
        idx = (cz[:, c, None, None] * ny + cy[:, :, None]) * nx + cx[:, None, :]
        np.add.at(mesh.reshape(-1), idx.ravel(), w.ravel())
    return mesh


def mesh_potential(rho, G):
    """phi_mesh = M * irfft(G * rfft(rho)) (unnormalised inverse DFT)."""
    nz, ny, nx = rho.shape
    rk = np.fft.rfftn(rho)
    phi = np.fft.irfftn(rk * G, s=rho.shape, axes=(0, 1, 2)) * rho.size
    return phi, rk


def interpolate(pos, q, phi, params):
    """Per-particle potential phi_i and mesh force F_i = -q_i grad phi."""
    nx, ny, nz = params.mesh
    Lx, Ly, Lz = params.box
    P = params.P
    g = grid_coords(pos, params.box, params.mesh)
    i0, t = stencil_origin(g, P)
    W = [params.window.weights(t[:, d]) for d in range(3)]
    dW = [params.window.dweights(t[:, d]) for d in range(3)]
    a = np.arange(P)
    cx = np.mod(i0[:, 0:1] + a, nx)
    cy = np.mod(i0[:, 1:2] + a, ny)
    cz = np.mod(i0[:, 2:3] + a, nz)
    N = pos.shape[0]
    pot = np.zeros(N)
    grad = np.zeros((N, 3))
    flat = phi.reshape(-1)
    for c in range(P):
        idx = (cz[:, c, None, None] * ny + cy[:, :, None]) * nx + cx[:, None, :]
        ph = flat[idx]  # [N, P(y), P(x)]
        pot += W[2][:, c] * np.einsum("nyx,ny,nx->n", ph, W[1], W[0])
        # dW/dt with dt/dg = -1 and dg/dr = n/L: d/dr w = -(n/L) dW/dt
        grad[:, 0] += W[2][:, c] * np.einsum("nyx,ny,nx->n", ph, W[1], dW[0]) * (-nx / Lx)
        grad[:, 1] += W[2][:, c] * np.einsum("nyx,ny,nx->n", ph, dW[1], W[0]) * (-ny / Ly)
        grad[:, 2] += dW[2][:, c] * np.einsum("nyx,ny,nx->n", ph, W[1], W[0]) * (-nz / Lz)
    F = -q[:, None] * grad
    return pot, F


def kspace_virial(rk, params, G=None, B=None):
    """W_ab = sum_k E_k (delta_ab + B(k) k_a k_b), E_k from the mesh spectrum."""
    nx, ny, nz = params.mesh
    Lx, Ly, Lz = params.box
    G = influence(params) if G is None else G
    B = influence(params, "B") if B is None else B
    kx = 2 * math.pi * np.arange(nx // 2 + 1) / Lx
    ky = 2 * math.pi * np.fft.fftfreq(ny, 1.0 / ny) / Ly
    kz = 2 * math.pi * np.fft.fftfreq(nz, 1.0 / nz) / Lz
    KZ, KY, KX = np.meshgrid(kz, ky, kx, indexing="ij")
    mult = np.full(nx // 2 + 1, 2.0)
    mult[0] = 1.0
    if nx % 2 == 0:
        mult[-1] = 1.0
    Ek = 0.5 * G * np.abs(rk) ** 2 * mult[None, None, :]
    comps = [(KX, KX), (KX, KY), (KX, KZ), (KY, KY), (KY, KZ), (KZ, KZ)]
    diag = [True, False, False, True, False, True]
    return np.array([np.sum(Ek * ((1.0 if d else 0.0) + B * a * b)) for (a, b), d in zip(comps, diag)]), \
        float(np.sum(Ek))


def _per_particle_virial(N, i_idx, f, d):
    """HOOMD's per-particle virial: half of each listed pair's r_a F_b on
    the listing particle, [N, 6] in the order xx, xy, xz, yy, yz, zz."""
    comps = [(0, 0), (0, 1), (0, 2), (1, 1), (1, 2), (2, 2)]
    Wpp = np.zeros((N, 6))
    for k, (a, b) in enumerate(comps):
        np.add.at(Wpp[:, k], i_idx, 0.5 * f * d[:, a] * d[:, b])
    return Wpp


def pair_forces(pos, q, box, split, rcut, nl_head, nl_count, nl_list, per_particle=False):
    """Short-range term over a full CSR neighbour list (HOOMD layout:
    neighbours of i are nl_list[nl_head[i] : nl_head[i] + nl_count[i]]).

    Per pair (``EvaluatorPairPSWF::evalForceAndEnergy``,
    ``src/EvaluatorPairPSWF.h:274-295``): ``pair_eng = qiqj L(r)``,
    ``force_divr = qiqj (-dL/dr) / r`` with
    ``4 pi L = 1/r - Q(r^2/r_c^2)/r_c``.  Energy is split half per particle
    as HOOMD does. Returns (F[N,3], e[N], virial[6]) and, with
    per_particle, the per-particle virial [N, 6] as a fourth value.
    """
    pos = np.asarray(pos, dtype=np.float64)
    L = np.asarray(box, dtype=np.float64)
    N = pos.shape[0]
    cnt = np.asarray(nl_count, dtype=np.int64)
    i_idx = np.repeat(np.arange(N), cnt)
    starts = np.asarray(nl_head, dtype=np.int64)
    offs = np.arange(cnt.sum()) - np.repeat(np.cumsum(cnt) - cnt, cnt)
    j_idx = np.asarray(nl_list, dtype=np.int64)[np.repeat(starts, cnt) + offs]
    d = pos[i_idx] - pos[j_idx]
    d -= L * np.round(d / L)
    r2 = np.sum(d * d, -1)
    m = (r2 < rcut * rcut) & (r2 > 0)
    r = np.sqrt(np.where(m, r2, 1.0))
    u = r2 / (rcut * rcut)
    qq = q[i_idx] * q[j_idx]
    Lr = INV_4PI * (1.0 / r - split.Q(u) / rcut)
    fdr = INV_4PI * (1.0 / (r * r * r) + 2.0 * split.dQ(u) / rcut ** 3)
    e = np.where(m, qq * Lr, 0.0)
    f = np.where(m, qq * fdr, 0.0)
    F = np.zeros((N, 3))
    np.add.at(F, i_idx, f[:, None] * d)
    en = np.zeros(N)
    np.add.at(en, i_idx, 0.5 * e)
    W = 0.5 * np.einsum("p,pa,pb->ab", f, d, d)
    vir = np.array([W[0, 0], W[0, 1], W[0, 2], W[1, 1], W[1, 2], W[2, 2]])
    if per_particle:
        return F, en, vir, _per_particle_virial(N, i_idx, f, d)
    return F, en, vir


def exclusion_correction(pos, q, box, split, rcut, n_ex, ex_list, ex_pitch, per_particle=False):
    """Removes the mesh's long-range interaction of excluded pairs
    (``gpu_esp_fix_exclusions_kernel``, ``src/ESPForceComputeGPU.cu:391-471``).

    The mesh sums ``q_i q_j Phi(r)`` over every pair, with
    ``Phi = 1/(4 pi r) - L(r)``: ``Q(r^2/r_c^2) / (4 pi r_c)`` inside the
    cutoff, the bare ``1/(4 pi r)`` beyond it (the reference skips excluded
    pairs beyond r_c). Exclusions of particle i are
    ``ex_list[i * ex_pitch + k], k < n_ex[i]``, listed from both sides; each
    side takes half of the pair energy. Returns (F[N,3], e[N], virial[6])
    and, with per_particle, the per-particle virial [N, 6].
    """
    pos = np.asarray(pos, dtype=np.float64)
    L = np.asarray(box, dtype=np.float64)
    N = pos.shape[0]
    cnt = np.asarray(n_ex, dtype=np.int64)
    i_idx = np.repeat(np.arange(N), cnt)
    k_idx = np.arange(cnt.sum()) - np.repeat(np.cumsum(cnt) - cnt, cnt)
    j_idx = np.asarray(ex_list, dtype=np.int64)[i_idx * ex_pitch + k_idx]
    d = pos[i_idx] - pos[j_idx]
    d -= L * np.round(d / L)
    r2 = np.sum(d * d, -1)
    inside = r2 < rcut * rcut
    u = np.where(inside, r2 / (rcut * rcut), 0.0)
    r = np.sqrt(np.where(inside, 1.0, r2))
    phi = np.where(inside, INV_4PI * split.Q(u) / rcut, INV_4PI / r)
    # dPhi/dr / r
    dphi_r = np.where(inside, INV_4PI * 2.0 * split.dQ(u) / rcut ** 3, -INV_4PI / (r * r * r))
    qq = q[i_idx] * q[j_idx]
    f = qq * dphi_r  # correction force on i is +f d (minus the mesh's -dE/dr)
    F = np.zeros((N, 3))
    np.add.at(F, i_idx, f[:, None] * d)
    en = np.zeros(N)
    np.add.at(en, i_idx, -0.5 * qq * phi)
    W = 0.5 * np.einsum("p,pa,pb->ab", f, d, d)
    vir = np.array([W[0, 0], W[0, 1], W[0, 2], W[1, 1], W[1, 2], W[2, 2]])
    if per_particle:
        return F, en, vir, _per_particle_virial(N, i_idx, f, d)
    return F, en, vir


def molecule_exclusions(n_mol: int, per_mol: int):
    """Exclusions of rigid molecules of `per_mol` consecutive particles:
    every particle excludes the others of its molecule. Returns
    (n_ex[N], ex_list[N * (per_mol - 1)], ex_pitch)."""
    N = n_mol * per_mol
    pitch = per_mol - 1
    n_ex = np.full(N, pitch, dtype=np.uint32)
    ex = np.zeros(N * pitch, dtype=np.uint32)
    for i in range(N):
        m0 = (i // per_mol) * per_mol
        ex[i * pitch:(i + 1) * pitch] = [j for j in range(m0, m0 + per_mol) if j != i]
    return n_ex, ex, pitch


def remove_pairs(nlist, n_ex, ex_list, ex_pitch):
    """A CSR neighbour list without the excluded pairs (HOOMD's neighbour
    list leaves them out)."""
    head, cnt, lst = nlist
    excl = set()
    for i in range(len(n_ex)):
        for k in range(int(n_ex[i])):
            excl.add((i, int(ex_list[i * ex_pitch + k])))
    nh, nc, nl = [], [], []
    for i in range(len(head)):
        nh.append(len(nl))
        row = [int(j) for j in lst[head[i]:head[i] + cnt[i]] if (i, int(j)) not in excl]
        nl.extend(row)
        nc.append(len(row))
    return (np.array(nh, dtype=np.uint32), np.array(nc, dtype=np.uint32), np.array(nl, dtype=np.uint32))


def lj_forces(pos, box, nlist, eps, sigma, rcut):
    """Lennard-Jones 4 eps ((sigma/r)^12 - (sigma/r)^6), r < rcut, unshifted,
    over a full CSR neighbour list (the MD harness's core repulsion).
    Returns (F[N,3], e[N]) with half the pair energy per particle."""
    pos = np.asarray(pos, dtype=np.float64)
    L = np.asarray(box, dtype=np.float64)
    head, cnt, lst = nlist
    N = pos.shape[0]
    cnt = np.asarray(cnt, dtype=np.int64)
    i_idx = np.repeat(np.arange(N), cnt)
    offs = np.arange(cnt.sum()) - np.repeat(np.cumsum(cnt) - cnt, cnt)
    j_idx = np.asarray(lst, dtype=np.int64)[np.repeat(np.asarray(head, dtype=np.int64), cnt) + offs]
    d = pos[i_idx] - pos[j_idx]
    d -= L * np.round(d / L)
    r2 = np.sum(d * d, -1)
    m = (r2 < rcut * rcut) & (r2 > 0)
    s6 = np.where(m, (sigma * sigma / np.where(m, r2, 1.0)) ** 3, 0.0)
    fdr = np.where(m, 24.0 * eps * (2.0 * s6 * s6 - s6) / np.where(m, r2, 1.0), 0.0)
    F = np.zeros((N, 3))
    np.add.at(F, i_idx, fdr[:, None] * d)
    en = np.zeros(N)
    np.add.at(en, i_idx, 0.5 * 4.0 * eps * (s6 * s6 - s6))
    return F, en


def neighbor_list(pos, box, rlist):
    """Full CSR neighbour list of all pairs with r < rlist (minimum image).
    Rows are sorted by neighbour index. Returns (head, count, list)."""
    from scipy.spatial import cKDTree

    pos = np.asarray(pos, dtype=np.float64)
    L = np.asarray(box, dtype=np.float64)
    p = pos - L * np.floor(pos / L)
    p = np.minimum(p, np.nextafter(L, 0))
    tree = cKDTree(p, boxsize=L)
    pairs = tree.query_pairs(rlist, output_type="ndarray")
    N = pos.shape[0]
    ii = np.concatenate([pairs[:, 0], pairs[:, 1]])
    jj = np.concatenate([pairs[:, 1], pairs[:, 0]])
    order = np.lexsort((jj, ii))
    ii = ii[order]
    jj = jj[order]
    count = np.bincount(ii, minlength=N).astype(np.uint32)
    head = (np.cumsum(count) - count).astype(np.uint32)
    return head, count, jj.astype(np.uint32)


def self_energy(q, params):
    """-1/2 Lambda(0) sum q^2, Lambda(0) = Q(0)/(4 pi r_c) (stub in the
    reference: ``computePSWFSelfEnergyConst``, ``src/ESPForceCompute.cc:386-396``)."""
    return -0.5 * params.split.lambda0 * INV_4PI / params.rcut * float(np.sum(np.asarray(q) ** 2))


def background_energy(q, params):
    """Neutralising background -(Q^2/2V) int L d^3r, int L d^3r = r_c^2 m2 / 2."""
    V = float(np.prod(params.box))
    Q = float(np.sum(q))
    return -(Q * Q) / (2.0 * V) * (params.rcut ** 2 * params.split.m2 * 0.5)


def esp(pos, q, params, nlist=None, return_parts: bool = False, exclusions=None):
    """Full ESP evaluation in FP64: returns (E, F[N,3], virial[6]) and,
    with return_parts, a dict of the stage outputs. `exclusions` =
    (n_ex, ex_list, ex_pitch) applies the exclusion correction (the
    neighbour list must then leave the excluded pairs out)."""
    pos = np.asarray(pos, dtype=np.float64)
    q = np.asarray(q, dtype=np.float64)
    G = influence(params)
    rho = spread(pos, q, params)
    phi, rk = mesh_potential(rho, G)
    pot, Fm = interpolate(pos, q, phi, params)
    if nlist is None:
        nlist = neighbor_list(pos, params.box, params.rcut)
        if exclusions is not None:
            nlist = remove_pairs(nlist, *exclusions)
    Fp, ep, Wp = pair_forces(pos, q, params.box, params.split, params.rcut, *nlist)
    E_rec = 0.5 * float(np.sum(q * pot))
    E_self = self_energy(q, params)
    E_bg = background_energy(q, params)
    Wk, _ = kspace_virial(rk, params, G)
    Wk = Wk + np.array([1, 0, 0, 1, 0, 1.0]) * E_bg
    E = E_rec + float(np.sum(ep)) + E_self + E_bg
    F = Fm + Fp
    vir = Wk + Wp
    if exclusions is not None:
        Fx, ex_e, Wx = exclusion_correction(pos, q, params.box, params.split, params.rcut, *exclusions)
        F = F + Fx
        E += float(np.sum(ex_e))
        vir = vir + Wx
        ep = ep + ex_e
    if return_parts:
        return E, F, vir, dict(rho=rho, phi=phi, pot=pot, F_mesh=Fm, F_pair=Fp, e_pair=ep, E_rec=E_rec,
                               E_self=E_self, E_bg=E_bg, W_k=Wk, W_pair=Wp, G=G)
    return E, F, vir


def rel_rms(F, Fref):
    return float(np.sqrt(np.sum((F - Fref) ** 2) / np.sum(Fref ** 2)))
