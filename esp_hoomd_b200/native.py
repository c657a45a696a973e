"""Python handles over the native ESP contexts (device buffers are torch
CUDA tensors; torch is only the allocator and stream provider here)."""
from __future__ import annotations

import ctypes
from typing import Optional, Sequence, Tuple

import numpy as np
import torch

from . import _lib
from ._lib import EspInfo, EspParams, check, get_lib


def make_params(order: int = 8, rcut: float = 3.0, kappa: float = 0.0, mesh: Optional[Sequence[int]] = None,
                target_error: float = 1e-5, window_c: float = 0.0, window_degree: int = 0, tile: int = 0,
                threads_per_particle: int = 0, alpha: float = 0.0, n_table: int = 512,
                precision: int = 0, fft_mode: int = 0, interp_mode: int = 0) -> EspParams:
    p = EspParams()
    check(get_lib().esp_params_default(ctypes.byref(p)), "esp_params_default")
    p.order = int(order)
    p.rcut = float(rcut)
    p.kappa = float(kappa)
    p.alpha = float(alpha)
    p.n_table = int(n_table)
    if mesh is not None:
        p.nx, p.ny, p.nz = (int(m) for m in mesh)
    p.target_error = float(target_error)
    p.window_c = float(window_c)
    p.window_degree = int(window_degree)
    p.tile = int(tile)
    p.threads_per_particle = int(threads_per_particle)
    p.precision = int(precision)
    p.fft_mode = int(fft_mode)
    p.interp_mode = int(interp_mode)
    return p


def _ptr(t: Optional[torch.Tensor]):
    if t is None:
        return None
    if not t.is_cuda:
        raise ValueError("device tensor expected")
    if not t.is_contiguous():
        raise ValueError("contiguous tensor expected")
    return ctypes.c_void_p(t.data_ptr())


def _stream(stream=None):
    s = stream if stream is not None else torch.cuda.current_stream()
    return ctypes.c_void_p(s.cuda_stream)


def info_dict(inf: EspInfo) -> dict:
    return {f[0]: getattr(inf, f[0]) for f in EspInfo._fields_}


class Context:
    """One system (plain path): wraps esp_create / esp_compute."""

    def __init__(self, params: EspParams, box: Sequence[float], N: int):
        self._lib = get_lib()
        self._h = ctypes.c_void_p()
        self.params = params
        self.box = tuple(float(b) for b in box)
        check(self._lib.esp_create(ctypes.byref(params), *self.box, int(N), ctypes.byref(self._h)), "esp_create")

    def compute(self, pos4: torch.Tensor, q: torch.Tensor, force4: torch.Tensor, energy: Optional[torch.Tensor] = None,
                virial: Optional[torch.Tensor] = None, nlist=None, flags: int = _lib.ESP_ALL, stream=None) -> None:
        head, nn, nl = nlist if nlist is not None else (None, None, None)
        check(self._lib.esp_compute(self._h, _stream(stream), _ptr(pos4), _ptr(q), int(pos4.shape[0]), _ptr(head),
                                    _ptr(nn), _ptr(nl), _ptr(force4), _ptr(energy), _ptr(virial), int(flags)),
              "esp_compute")

    def compute_hoomd(self, pos4: torch.Tensor, q: torch.Tensor, force4: torch.Tensor, virial_pp: torch.Tensor,
                      external: torch.Tensor, nlist=None, flags: int = _lib.ESP_ALL, stream=None) -> None:
        """HOOMD ForceCompute outputs: force4 (m_force), virial_pp [6, pitch]
        float32 (m_virial), external [7] float64 (m_external_energy, then
        m_external_virial)."""
        head, nn, nl = nlist if nlist is not None else (None, None, None)
        if virial_pp.dim() != 2 or virial_pp.shape[0] != 6 or virial_pp.dtype != torch.float32:
            raise ValueError("virial_pp: float32 tensor of shape [6, pitch] expected")
        check(self._lib.esp_compute_hoomd(self._h, _stream(stream), _ptr(pos4), _ptr(q), int(pos4.shape[0]),
                                          _ptr(head), _ptr(nn), _ptr(nl), _ptr(force4), _ptr(virial_pp),
                                          int(virial_pp.shape[1]), _ptr(external), int(flags)), "esp_compute_hoomd")

    def compute_f64(self, pos4: torch.Tensor, q: torch.Tensor, force4: torch.Tensor,
                    energy: Optional[torch.Tensor] = None, virial: Optional[torch.Tensor] = None, nlist=None,
                    flags: int = _lib.ESP_ALL, stream=None) -> None:
        """FP64 evaluation (float64 tensors; context created with precision=1)."""
        head, nn, nl = nlist if nlist is not None else (None, None, None)
        check(self._lib.esp_compute_f64(self._h, _stream(stream), _ptr(pos4), _ptr(q), int(pos4.shape[0]),
                                        _ptr(head), _ptr(nn), _ptr(nl), _ptr(force4), _ptr(energy), _ptr(virial),
                                        int(flags)), "esp_compute_f64")

    def spread(self, pos4: torch.Tensor, q: torch.Tensor, stream=None) -> torch.Tensor:
        """Charge mesh rho[nz, ny, nx] (float64) of the bin+sort+spread stages."""
        inf = self.info()
        rho = torch.empty((inf["nz"], inf["ny"], inf["nx"]), dtype=torch.float64, device=pos4.device)
        check(self._lib.esp_spread(self._h, _stream(stream), _ptr(pos4), _ptr(q), int(pos4.shape[0]), _ptr(rho)),
              "esp_spread")
        return rho

    def sort_state(self, N: int, device="cuda", stream=None):
        """(key[N], perm[N]) of the last call (uint32 stored in int32 tensors)."""
        key = torch.empty(N, dtype=torch.int32, device=device)
        perm = torch.empty(N, dtype=torch.int32, device=device)
        check(self._lib.esp_get_sort(self._h, _stream(stream), _ptr(key), _ptr(perm)), "esp_get_sort")
        return key, perm

    def potential(self, stream=None) -> torch.Tensor:
        inf = self.info()
        phi = torch.empty((inf["nz"], inf["ny"], inf["nx"]), dtype=torch.float32, device="cuda")
        check(self._lib.esp_get_potential(self._h, _stream(stream), _ptr(phi)), "esp_get_potential")
        return phi

    def set_params(self, params: EspParams) -> None:
        self.params = params
        check(self._lib.esp_set_params(self._h, ctypes.byref(params)), "esp_set_params")

    def set_box(self, box: Sequence[float]) -> None:
        self.box = tuple(float(b) for b in box)
        check(self._lib.esp_set_box(self._h, *self.box), "esp_set_box")

    def invalidate(self) -> None:
        check(self._lib.esp_invalidate(self._h), "esp_invalidate")

    def set_exclusions(self, n_ex: Optional[torch.Tensor], ex_list: Optional[torch.Tensor] = None,
                       ex_pitch: int = 0) -> None:
        """Excluded pairs (device uint32 arrays, row i = ex_list[i * ex_pitch:]); None clears."""
        self._ex = (n_ex, ex_list)
        check(self._lib.esp_set_exclusions(self._h, _ptr(n_ex), _ptr(ex_list), int(ex_pitch)), "esp_set_exclusions")

    def info(self) -> dict:
        inf = EspInfo()
        check(self._lib.esp_get_info(self._h, ctypes.byref(inf)), "esp_get_info")
        return info_dict(inf)

    def close(self) -> None:
        if self._h:
            self._lib.esp_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Batch:
    """Many independent systems evaluated by one launch per stage."""

    def __init__(self, params: EspParams, N: Sequence[int], boxes: Sequence[Sequence[float]],
                 meshes: Optional[Sequence[Sequence[int]]] = None):
        self._lib = get_lib()
        self._h = ctypes.c_void_p()
        self.N = np.asarray(N, dtype=np.int32)
        self.boxes = np.asarray(boxes, dtype=np.float64).reshape(-1, 3)
        self.offsets = np.concatenate([[0], np.cumsum(self.N)]).astype(np.int64)
        m = None if meshes is None else np.ascontiguousarray(np.asarray(meshes, dtype=np.int32).reshape(-1, 3))
        self._m = m
        check(self._lib.esp_batch_create(ctypes.byref(params), int(self.N.size),
                                         self.N.ctypes.data_as(ctypes.c_void_p),
                                         self.boxes.ctypes.data_as(ctypes.c_void_p),
                                         None if m is None else m.ctypes.data_as(ctypes.c_void_p),
                                         ctypes.byref(self._h)), "esp_batch_create")

    @property
    def nsys(self) -> int:
        return int(self.N.size)

    @property
    def total(self) -> int:
        return int(self.offsets[-1])

    def compute(self, pos4, q, force4, energy=None, virial=None, nlist=None, flags: int = _lib.ESP_ALL,
                stream=None) -> None:
        head, nn, nl = nlist if nlist is not None else (None, None, None)
        check(self._lib.esp_batch_compute(self._h, _stream(stream), _ptr(pos4), _ptr(q), _ptr(head), _ptr(nn),
                                          _ptr(nl), _ptr(force4), _ptr(energy), _ptr(virial), int(flags)),
              "esp_batch_compute")

    def build_nlist(self, pos4, rlist: float, cap: int, head, nn, nl, stream=None) -> None:
        """HOOMD-layout neighbour rows into the caller's arrays. Does not
        synchronise: a row overflow is reported by nlist_check and by the
        next compute / md_run over these rows."""
        check(self._lib.esp_batch_build_nlist(self._h, _stream(stream), _ptr(pos4), float(rlist), int(cap),
                                              _ptr(head), _ptr(nn), _ptr(nl)), "esp_batch_build_nlist")

    def nlist_check(self) -> int:
        """Waits for the last build_nlist; raises EspError (ESP_ERR_OVERFLOW)
        if a row exceeded its capacity (then n_neigh holds the needed counts);
        returns 0."""
        need = ctypes.c_int(0)
        check(self._lib.esp_batch_nlist_check(self._h, ctypes.byref(need)), "esp_batch_nlist_check")
        return int(need.value)

    def build_pairlist(self, pos4, rlist: float, cap: int = 256, stream=None) -> None:
        """Builds the library-owned pair list (all pairs with r < rlist, rows
        in cell order); compute / md_run without a neighbour list use it.
        Does not synchronise: a row overflow is reported by a later call."""
        check(self._lib.esp_batch_build_pairlist(self._h, _stream(stream), _ptr(pos4), float(rlist), int(cap)),
              "esp_batch_build_pairlist")

    def device_errors(self) -> int:
        """Error word of the batch's kernels since the last call (bit 0: a
        TMA-staged interpolation tile timed out); synchronises."""
        f = ctypes.c_int(0)
        check(self._lib.esp_batch_device_errors(self._h, ctypes.byref(f)), "esp_batch_device_errors")
        return int(f.value)

    def pairlist_check(self) -> int:
        """Waits for the last pair-list build; raises EspError (ESP_ERR_OVERFLOW)
        if a row exceeded its capacity; returns 0."""
        need = ctypes.c_int(0)
        check(self._lib.esp_batch_pairlist_check(self._h, ctypes.byref(need)), "esp_batch_pairlist_check")
        return int(need.value)

    def nve_step1(self, pos4, vel4, force4, dt: float, stream=None) -> None:
        check(self._lib.esp_batch_nve_step1(self._h, _stream(stream), _ptr(pos4), _ptr(vel4), _ptr(force4),
                                            float(dt)), "esp_batch_nve_step1")

    def nve_step2(self, vel4, force4, dt: float, pos4=None, stream=None) -> None:
        """Second half kick; pos4 (the current positions) is needed with rigid molecules."""
        check(self._lib.esp_batch_nve_step2(self._h, _stream(stream), _ptr(pos4), _ptr(vel4), _ptr(force4),
                                            float(dt)), "esp_batch_nve_step2")

    def set_rigid_water(self, first, count, d_oh: float, d_hh: float) -> None:
        """Rigid (O, H, H) molecules: system s has count[s] consecutive triples
        from local particle first[s]; None clears."""
        if first is None:
            check(self._lib.esp_batch_set_rigid_water(self._h, None, None, 0.0, 0.0), "esp_batch_set_rigid_water")
            return
        f = np.ascontiguousarray(np.asarray(first, dtype=np.int32))
        c = np.ascontiguousarray(np.asarray(count, dtype=np.int32))
        check(self._lib.esp_batch_set_rigid_water(self._h, f.ctypes.data_as(ctypes.c_void_p),
                                                  c.ctypes.data_as(ctypes.c_void_p), float(d_oh), float(d_hh)),
              "esp_batch_set_rigid_water")

    def md_run(self, pos4, vel4, q, force4, energy, virial, nlist, nsteps: int, dt: float, use_graph: bool = True,
               stream=None) -> None:
        """nlist = (head, n_neigh, nlist) or None for the library's pair list."""
        head, nn, nl = nlist if nlist is not None else (None, None, None)
        check(self._lib.esp_batch_md_run(self._h, _stream(stream), _ptr(pos4), _ptr(vel4), _ptr(q), _ptr(head),
                                         _ptr(nn), _ptr(nl), _ptr(force4), _ptr(energy), _ptr(virial), int(nsteps),
                                         float(dt), int(bool(use_graph))), "esp_batch_md_run")

    def md_run_f64(self, pos4, vel4, q, force4, energy, virial, nlist, nsteps: int, dt: float,
                   lj: Optional[Tuple[float, float, float]] = None, use_graph: bool = True, stream=None) -> None:
        """FP64 velocity-Verlet steps (float64 tensors) over nlist = (head,
        n_neigh, nlist); lj = (epsilon, sigma, r_cut) adds the Lennard-Jones
        core to every step's forces and energy."""
        head, nn, nl = nlist
        eps, sig, rc = lj if lj is not None else (0.0, 0.0, 0.0)
        check(self._lib.esp_batch_md_run_f64(self._h, _stream(stream), _ptr(pos4), _ptr(vel4), _ptr(q), _ptr(head),
                                             _ptr(nn), _ptr(nl), _ptr(force4), _ptr(energy), _ptr(virial),
                                             int(nsteps), float(dt), float(eps), float(sig), float(rc),
                                             int(bool(use_graph))), "esp_batch_md_run_f64")

    def set_exclusions(self, n_ex: Optional[torch.Tensor], ex_list: Optional[torch.Tensor] = None,
                       ex_pitch: int = 0) -> None:
        """Excluded pairs of all systems (rows by concatenated index, local
        excluded indices); None clears."""
        self._ex = (n_ex, ex_list)
        check(self._lib.esp_batch_set_exclusions(self._h, _ptr(n_ex), _ptr(ex_list), int(ex_pitch)),
              "esp_batch_set_exclusions")

    def autotune(self, pos4, q, nlist=None, flags: int = _lib.ESP_ALL, reps: int = 3, stream=None) -> dict:
        """Times candidate plans on these inputs and keeps the fastest; returns
        the chosen knobs and the per-candidate milliseconds per evaluation."""
        head, nn, nl = nlist if nlist is not None else (None, None, None)
        chosen = EspParams()
        trials = np.zeros(16, dtype=np.float64)
        check(self._lib.esp_batch_autotune(self._h, _stream(stream), _ptr(pos4), _ptr(q), _ptr(head), _ptr(nn),
                                           _ptr(nl), int(flags), int(reps), ctypes.byref(chosen),
                                           trials.ctypes.data_as(ctypes.c_void_p), int(trials.size)),
              "esp_batch_autotune")
        return {"tile": chosen.tile, "threads_per_particle": chosen.threads_per_particle,
                "fft_mode": chosen.fft_mode, "interp_mode": chosen.interp_mode,
                "trial_ms": [float(t) for t in trials if t > 0]}

    def compute_f64(self, pos4, q, force4, energy=None, virial=None, nlist=None, flags: int = _lib.ESP_ALL,
                    stream=None) -> None:
        """FP64 evaluation (float64 tensors; batch created with precision=1)."""
        head, nn, nl = nlist if nlist is not None else (None, None, None)
        check(self._lib.esp_batch_compute_f64(self._h, _stream(stream), _ptr(pos4), _ptr(q), _ptr(head), _ptr(nn),
                                              _ptr(nl), _ptr(force4), _ptr(energy), _ptr(virial), int(flags)),
              "esp_batch_compute_f64")

    def lj(self, pos4, nlist, epsilon: float, sigma: float, r_cut: float, force4, energy=None, stream=None) -> None:
        """Adds Lennard-Jones forces/energies (float32 or float64 tensors)."""
        head, nn, nl = nlist
        fn = self._lib.esp_batch_lj_f64 if pos4.dtype == torch.float64 else self._lib.esp_batch_lj
        check(fn(self._h, _stream(stream), _ptr(pos4), _ptr(head), _ptr(nn), _ptr(nl), float(epsilon), float(sigma),
                 float(r_cut), _ptr(force4), _ptr(energy)), "esp_batch_lj")

    def nve_step1_f64(self, pos4, vel4, force4, dt: float, stream=None) -> None:
        check(self._lib.esp_batch_nve_step1_f64(self._h, _stream(stream), _ptr(pos4), _ptr(vel4), _ptr(force4),
                                                float(dt)), "esp_batch_nve_step1_f64")

    def nve_step2_f64(self, vel4, force4, dt: float, pos4=None, stream=None) -> None:
        check(self._lib.esp_batch_nve_step2_f64(self._h, _stream(stream), _ptr(pos4), _ptr(vel4), _ptr(force4),
                                                float(dt)), "esp_batch_nve_step2_f64")

    def set_timing(self, on: bool) -> None:
        check(self._lib.esp_batch_set_timing(self._h, int(bool(on))), "esp_batch_set_timing")

    def stage_times(self) -> dict:
        """{stage: (total ms, launches)} since timing was enabled or last read."""
        ms = np.zeros(len(_lib.STAGES), dtype=np.float64)
        cnt = np.zeros(len(_lib.STAGES), dtype=np.int64)
        check(self._lib.esp_batch_stage_times(self._h, ms.ctypes.data_as(ctypes.c_void_p),
                                              cnt.ctypes.data_as(ctypes.c_void_p)), "esp_batch_stage_times")
        return {k: (float(ms[i]), int(cnt[i])) for i, k in enumerate(_lib.STAGES)}

    def info(self, s: int) -> dict:
        inf = EspInfo()
        check(self._lib.esp_batch_get_info(self._h, int(s), ctypes.byref(inf)), "esp_batch_get_info")
        return info_dict(inf)

    def close(self) -> None:
        if self._h:
            self._lib.esp_batch_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def _host_ptr(a, dtype, count: int, name: str):
    """Address of a contiguous host array (numpy, or a CPU torch tensor such
    as a pinned one) holding at least `count` elements of `dtype`."""
    if a is None:
        return None
    if isinstance(a, torch.Tensor):
        if a.is_cuda or not a.is_contiguous() or a.numel() < count:
            raise ValueError("%s: contiguous host tensor of %d elements expected" % (name, count))
        return ctypes.c_void_p(a.data_ptr())
    if not (isinstance(a, np.ndarray) and a.dtype == dtype and a.flags["C_CONTIGUOUS"] and a.size >= count):
        raise ValueError("%s: contiguous %s array of %d elements expected" % (name, np.dtype(dtype).name, count))
    return ctypes.c_void_p(a.ctypes.data)


class Server:
    """Continuous-batching request server over the C ABI (esp_server_*).

    Host buffers passed to ``submit`` are referenced until ``close`` (the
    server reads and writes them asynchronously)."""

    def __init__(self, params: EspParams, hbm_budget: int = 4 << 30, max_systems: int = 512,
                 max_particles: int = 262144):
        self._lib = get_lib()
        self._h = ctypes.c_void_p()
        cfg = _lib.EspServerConfig(params=params, hbm_budget=int(hbm_budget), max_systems=int(max_systems),
                                   max_particles=int(max_particles))
        check(self._lib.esp_server_create(ctypes.byref(cfg), ctypes.byref(self._h)), "esp_server_create")
        self._keep = []

    def submit(self, pos4, charge, box: Sequence[float], rcut: float, vel4=None, nsteps: int = 10,
               dt: float = 0.002, skin: float = 0.4, arrival: float = 0.0, nlist_cap: int = 0, out_pos4=None,
               out_vel4=None, out_force4=None, out_energy=None, rigid_water=None) -> int:
        """rigid_water = (d_oh, d_hh): the system is (O, H, H) triples kept rigid."""
        N = int(len(charge))
        r = _lib.EspRequest()
        r.N = N
        r.Lx, r.Ly, r.Lz = (float(b) for b in box)
        r.rcut = float(rcut)
        r.skin = float(skin)
        r.nlist_cap = int(nlist_cap)
        r.nsteps = int(nsteps)
        r.dt = float(dt)
        r.arrival = float(arrival)
        r.pos4 = _host_ptr(pos4, np.float32, 4 * N, "pos4")
        r.vel4 = _host_ptr(vel4, np.float32, 4 * N, "vel4")
        r.charge = _host_ptr(charge, np.float32, N, "charge")
        r.out_pos4 = _host_ptr(out_pos4, np.float32, 4 * N, "out_pos4")
        r.out_vel4 = _host_ptr(out_vel4, np.float32, 4 * N, "out_vel4")
        r.out_force4 = _host_ptr(out_force4, np.float32, 4 * N, "out_force4")
        r.out_energy = _host_ptr(out_energy, np.float64, 1, "out_energy")
        if rigid_water is not None:
            r.rigid_doh, r.rigid_dhh = (float(v) for v in rigid_water)
        rid = ctypes.c_longlong()
        check(self._lib.esp_server_submit(self._h, ctypes.byref(r), ctypes.byref(rid)), "esp_server_submit")
        self._keep.append((pos4, vel4, charge, out_pos4, out_vel4, out_force4, out_energy))
        return int(rid.value)

    def start(self) -> None:
        check(self._lib.esp_server_start(self._h), "esp_server_start")

    def status(self, rid: int) -> dict:
        s = _lib.EspRequestStatus()
        check(self._lib.esp_server_status(self._h, int(rid), ctypes.byref(s)), "esp_server_status")
        return {f[0]: getattr(s, f[0]) for f in _lib.EspRequestStatus._fields_}

    def wait_all(self, timeout: float = 600.0) -> None:
        check(self._lib.esp_server_wait_all(self._h, float(timeout)), "esp_server_wait_all")

    def stats(self) -> dict:
        s = _lib.EspServerStats()
        check(self._lib.esp_server_get_stats(self._h, ctypes.byref(s)), "esp_server_get_stats")
        return {f[0]: getattr(s, f[0]) for f in _lib.EspServerStats._fields_}

    def close(self) -> None:
        if self._h:
            self._lib.esp_server_destroy(self._h)
            self._h = ctypes.c_void_p()
        self._keep = []

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def pswf_eval_pairs(rsq: torch.Tensor, qiqj: torch.Tensor, rcut: float, table, stream=None):
    """Reference-format evaluator over n pairs on the GPU (FP64).

    ``table`` holds device float64 tensors screen, dscreen, r_lo, dr_inv.
    Returns (force_divr, pair_eng, evaluated)."""
    n = int(rsq.numel())
    fd = torch.empty(n, dtype=torch.float64, device=rsq.device)
    pe = torch.empty_like(fd)
    ev = torch.empty(n, dtype=torch.int32, device=rsq.device)
    screen, dscreen, r_lo, dr_inv = table
    check(get_lib().esp_pswf_eval_pairs(_stream(stream), n, _ptr(rsq), _ptr(qiqj), float(rcut), int(r_lo.numel()),
                                        _ptr(screen), _ptr(dscreen), _ptr(r_lo), _ptr(dr_inv), _ptr(fd), _ptr(pe),
                                        _ptr(ev)), "esp_pswf_eval_pairs")
    return fd, pe, ev
