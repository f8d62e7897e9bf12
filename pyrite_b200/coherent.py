"""Coherent (field-sum) CXR: the per-row field reduction on the device.

The reference's coherent route (``mc_cxr_spectrum(..., coherent=True)``,
``pyrite/montecarlo/spectrum/cxr/_batched.py:1029-1240``) turns every
(segment, reflection row) pair into a line record -- the ``per_cxr`` tuple of
``cxr/_batched.py:646-660`` -- and then reduces each row separately: the
complex field of both polarisations summed over the row's lines at every
output energy, squared, weighted by the row's mosaic weight and summed over
rows (``cxr/_batched_finalize.py:209-243``; its CUDA form
``run_coherent_reduction_kernel``, ``coherent_jit_kernel.py:716``). This module
hands that reduction to ``pb_coherent_reduce``: every row in one call, FP64
phases, a deterministic FP64 row sum.

``coherent_reduce`` takes the records of all rows at once;
``run_coherent_reduction_kernel`` keeps the reference's one-row signature
(vacuum sinc, in-medium phase, formation factor and sinc window as optional
groups, with the same pairing rules and errors). ``coherent_records`` builds
the records themselves on the device from a segment list
(``pb_coherent_records``, the reference's record prologue
``cxr/_batched.py:561-660``), and ``coherent_route_spectrum`` runs the whole
route, segments to spectrum.
"""

from __future__ import annotations

import ctypes as C

import numpy as np
import torch

from . import _lib as L
from .api import _device, _Holder, _stream_ptr

# Line record fields, in the order of cxr/_batched.py:646-660 (the emitting
# electron id, which only the decoherence blend reads, is not needed).
RECORD_FIELDS = ("E_vac", "a_vac", "phase_slope", "g_phase", "cs_re", "cs_im", "cp_re", "cp_im",
                 "L_esc", "half_dL", "apb", "bma", "q")


def _work(h: _Holder, n_row: int, n_line: int, n_E: int, blend: bool = False):
    lib = L.load()
    nbytes = C.c_uint64()
    if blend:
        L.check(lib.pb_coherent_blend_work_size(n_row, n_line, n_E, C.byref(nbytes)), "pb_coherent_blend_work_size")
    else:
        L.check(lib.pb_coherent_work_size(n_row, n_line, n_E, C.byref(nbytes)), "pb_coherent_work_size")
    # torch's caching allocator hands out 512-byte aligned blocks
    return h.empty((max(int(nbytes.value), 1),), torch.uint8), int(nbytes.value)


def coherent_reduce(records, row_count, row_weight, E_grid_eV, delta_omega, *, scale=1.0, sinc_cutoff=None,
                    spec=None, device=None, stream=None, status=None, elec_id=None, F_row=None) -> torch.Tensor:
    """``spec += scale * sum_rows w_r (|F_sigma|^2 + |F_pi|^2)`` on the device.

    ``records`` maps ``RECORD_FIELDS`` to per-line arrays (numpy or tensors),
    laid out row after row; ``row_count[r]`` lines belong to row ``r``, whose
    intensity is weighted by ``row_weight[r]``. ``delta_omega`` is
    ``(1 - Re n(E)) omega(E)`` on ``E_grid_eV`` [1/Angstrom]. Returns the FP64
    device spectrum (``spec`` when given, accumulated into).

    With ``elec_id`` (the emitting electron of every line, contiguous and
    nondecreasing inside a row) and ``F_row`` [n_row, n_E] (the rows'
    decoherence factors, ``decoherence_factor``), each row is the
    sampled-bunch blend ``F flat + (1 - F) grouped`` of its all-electron
    field and its per-electron squared fields (``pb_coherent_blend``).
    """
    dev = _device(device)
    h = _Holder(dev)
    row_count = np.asarray(row_count, dtype=np.int64)
    if row_count.ndim != 1 or row_count.size < 1 or np.any(row_count < 0):
        raise ValueError("row_count must be a nonempty 1-D array of nonnegative counts")
    n_row = int(row_count.size)
    n_line = int(row_count.sum())
    E = h.f64(E_grid_eV)
    n_E = int(E.numel())
    dom = h.f64(delta_omega)
    if int(dom.numel()) != n_E:
        raise ValueError("delta_omega must have one entry per energy")
    w = h.f64(row_weight)
    if int(w.numel()) != n_row:
        raise ValueError("row_weight must have one entry per row")
    fields = {}
    for name in RECORD_FIELDS:
        t = h.f64(records[name]).reshape(-1)
        if int(t.numel()) != n_line:
            raise ValueError(f"record field {name!r} has {int(t.numel())} lines, the rows hold {n_line}")
        fields[name] = t
    row_off = h.typed(np.concatenate([[0], np.cumsum(row_count)]).astype(np.int64), torch.int64)
    if spec is None:
        spec = h.zeros((n_E,), torch.float64)
    elif spec.dtype != torch.float64 or spec.device != dev or int(spec.numel()) != n_E or not spec.is_contiguous():
        raise ValueError("spec must be a contiguous float64 tensor on the device with one entry per energy")
    blend = elec_id is not None or F_row is not None
    if blend:
        if elec_id is None or F_row is None:
            raise ValueError("the decoherence blend needs both elec_id and F_row")
        eid = h.typed(np.asarray(elec_id, dtype=np.int64).reshape(-1) if not torch.is_tensor(elec_id)
                      else elec_id.reshape(-1), torch.int64)
        if int(eid.numel()) != n_line:
            raise ValueError("elec_id must have one entry per line")
        F = h.f64(F_row).reshape(-1)
        if int(F.numel()) != n_row * n_E:
            raise ValueError("F_row must be [n_row, n_E]")
    work, nbytes = _work(h, n_row, n_line, n_E, blend)
    a = L.PbCoherentArgs()
    a.n_row, a.n_E, a.n_line = n_row, n_E, n_line
    a.row_off, a.row_weight, a.E, a.delta_omega = (t.data_ptr() for t in (row_off, w, E, dom))
    for name in RECORD_FIELDS:
        setattr(a, name, fields[name].data_ptr())
    a.scale = float(scale)
    a.sinc_cutoff = 0.0 if sinc_cutoff is None else float(sinc_cutoff)
    a.spec = spec.data_ptr()
    a.work, a.work_bytes = work.data_ptr(), nbytes
    a.status = None if status is None else status.data_ptr()
    if blend:
        b = L.PbCoherentBlendArgs()
        b.base = a
        b.elec_id, b.F_row = eid.data_ptr(), F.data_ptr()
        L.check(L.load().pb_coherent_blend(C.byref(b), _stream_ptr(stream)), "pb_coherent_blend")
    else:
        L.check(L.load().pb_coherent_reduce(C.byref(a), _stream_ptr(stream)), "pb_coherent_reduce")
    if stream is not None:
        # freed on torch's current stream: keep the blocks until the call has run
        for t in h.keep:
            t.record_stream(stream)
    return spec


def coherent_records(segments, E_grid_eV, *, tables, rows, n_hat, device=None, stream=None, with_electrons=False):
    """The coherent route's per-row line records of one detector direction,
    built on the device from ``segments`` (the reference's segment dict with
    ``thickness_ang``, ``Ne`` and optional ``t_ang`` start ages) by
    ``pb_coherent_records``: ``(records, row_count)``, ``records`` mapping
    ``RECORD_FIELDS`` to FP64 device tensors laid out row after row (each row
    its kept pairs in segment order), ``row_count`` a numpy array. ``rows``:
    ``tables.ReflectionRows`` with one direction; ``tables``: ``LineTables``;
    ``E_grid_eV`` sets the keep window as the incoherent scorer's.
    ``with_electrons`` adds ``records["elec_id"]``, each record's electron."""
    from .api import _fill_tables, _ptr, _segments_on_device
    from .tables import line_keep_window

    dev = _device(device)
    lib = L.load()
    h = _Holder(dev)
    seg = _segments_on_device(h, segments)
    n_g = int(rows.G.shape[0])
    E_grid = np.asarray(E_grid_eV, dtype=np.float64)
    lo_keep, hi_keep = line_keep_window(E_grid)
    a = L.PbCoherentRecordsArgs()
    c = a.cxr
    c.precision = L.PB_FP64
    c.n_dir = 1
    nh = np.asarray(n_hat, dtype=float).reshape(3)
    c.n_hat = _ptr(h.f64(nh / np.linalg.norm(nh)))
    c.thickness = float(segments["thickness_ang"])
    c.Ne = int(segments["Ne"])
    c.n_seg = seg["n"]
    c.r_mid, c.v_hat, c.L = _ptr(seg["r_mid"]), _ptr(seg["v_hat"]), _ptr(seg["L"])
    c.E_keV, c.elec_id = _ptr(seg["E"]), _ptr(seg["elec_id"])
    t = _fill_tables(h, rows, tables, lo_keep, hi_keep)
    t.ES = _ptr(h.f64(np.asarray(rows.ES).reshape(-1, n_g, 3)[0]))
    t.EP = _ptr(h.f64(np.asarray(rows.EP).reshape(-1, n_g, 3)[0]))
    c.tables = t
    a.cxr = c
    t_ang = segments.get("t_ang")
    a.t_start = _ptr(h.f64(t_ang)) if t_ang is not None else None
    cap = max(1, seg["n"] * n_g)
    a.capacity = cap
    rec = {k: torch.empty(cap, dtype=torch.float64, device=dev) for k in RECORD_FIELDS}
    for k in RECORD_FIELDS:
        setattr(a, k, rec[k].data_ptr())
    if with_electrons:
        rec["elec_id"] = torch.empty(cap, dtype=torch.int64, device=dev)
        a.elec_out = rec["elec_id"].data_ptr()
    row_off = h.zeros(n_g + 1, torch.int64)
    a.row_off = row_off.data_ptr()
    nbytes = C.c_uint64()
    L.check(lib.pb_coherent_records_work_size(seg["n"], n_g, C.byref(nbytes)), "pb_coherent_records_work_size")
    work = h.empty((max(int(nbytes.value), 1),), torch.uint8)
    a.work, a.work_bytes = work.data_ptr(), int(nbytes.value)
    status = h.zeros(1, torch.int32)
    a.status = status.data_ptr()
    L.check(lib.pb_coherent_records(C.byref(a), _stream_ptr(stream)), "pb_coherent_records")
    off = row_off.cpu().numpy()
    if int(status.item()) != 0:
        raise L.PyriteB200Error(f"pb_coherent_records: device status {int(status.item())}")
    n_line = int(off[-1])
    return {k: v[:n_line] for k, v in rec.items()}, np.diff(off)


def coherent_route_spectrum(segments, E_grid_eV, delta_omega, *, tables, rows, n_hat, sinc_cutoff=None,
                            device=None) -> np.ndarray:
    """The coherent route end to end on the device for one direction:
    records from the segments (``coherent_records``), every row reduced with
    its mosaic weight (``pb_coherent_reduce``), divided by the electron
    count -- [photons/eV/sr/electron] as the reference's coherent
    ``mc_cxr_spectrum`` returns it (``cxr/_spectrum.py:285-318``)."""
    rec, cnt = coherent_records(segments, E_grid_eV, tables=tables, rows=rows, n_hat=n_hat, device=device)
    return coherent_spectrum(rec, cnt, np.asarray(rows.WM, dtype=float).reshape(-1), E_grid_eV, delta_omega,
                             int(segments["Ne"]), sinc_cutoff=sinc_cutoff, device=device)


def coherent_spectrum(records, row_count, row_weight, E_grid_eV, delta_omega, Ne, *, sinc_cutoff=None,
                      device=None) -> np.ndarray:
    """The coherent route's spectrum per electron [photons/eV/sr/electron],
    as ``_finalize_spectrum`` returns it (``cxr/_spectrum.py:285-318``)."""
    if Ne < 1:
        raise ValueError("Ne must be >= 1")
    spec = coherent_reduce(records, row_count, row_weight, E_grid_eV, delta_omega, scale=1.0 / Ne,
                           sinc_cutoff=sinc_cutoff, device=device)
    return spec.cpu().numpy()


def coherent_route_spectrum_streamed(segments, E_grid_eV, delta_omega, *, tables, rows, n_hat,
                                    block_segments=1 << 16, sinc_cutoff=None, decoherence=None,
                                    device=None) -> np.ndarray:
    """The coherent route over segment blocks, as the reference's streamed
    field-plane route does (``coherent_stream_jit_kernel.py``): each block's
    records (``coherent_records``) are folded into persistent FP64 field
    planes per row (``pb_coherent_accumulate``), which are squared and
    weighted once at the end (``pb_coherent_finalize``), so memory holds one
    block's records, not the whole run's. Blocks end on electron boundaries
    (the segments must be in electron order). ``decoherence`` =
    ``dict(A_pop=, xy0_pop=, omega=)`` applies the sampled-bunch blend with
    the rows' factors, the per-electron fields accumulated beside the flat
    ones. Per electron, as ``coherent_route_spectrum``."""
    dev = _device(device)
    lib = L.load()
    h = _Holder(dev)
    eid = np.asarray(segments["elec_id"]).reshape(-1)
    n = int(eid.size)
    if np.any(np.diff(eid) < 0):
        raise ValueError("the streamed route needs the segments in electron order")
    starts = [0]
    while starts[-1] < n:
        b = min(starts[-1] + int(block_segments), n)
        while 0 < b < n and eid[b] == eid[b - 1]:
            b += 1
        starts.append(b)
    E = h.f64(E_grid_eV)
    dom = h.f64(delta_omega)
    n_E, n_row = int(E.numel()), int(np.asarray(rows.G).reshape(-1, 3).shape[0])
    w = h.f64(np.asarray(rows.WM, dtype=float).reshape(-1))
    fields = h.zeros((n_row * 4 * n_E,), torch.float64)
    power = h.zeros((n_row * n_E,), torch.float64) if decoherence is not None else None
    arrays = {k: v for k, v in segments.items() if k not in ("Ne", "thickness_ang")}
    for s0, s1 in zip(starts[:-1], starts[1:]):
        sub = {k: np.asarray(v)[s0:s1] for k, v in arrays.items()}
        sub["Ne"], sub["thickness_ang"] = segments["Ne"], segments["thickness_ang"]
        rec, cnt = coherent_records(sub, E_grid_eV, tables=tables, rows=rows, n_hat=n_hat, device=dev,
                                    with_electrons=decoherence is not None)
        n_line = int(cnt.sum())
        if n_line == 0:
            continue
        a = L.PbCoherentStreamArgs()
        b = a.base
        b.n_row, b.n_E, b.n_line = n_row, n_E, n_line
        row_off = h.typed(np.concatenate([[0], np.cumsum(cnt)]).astype(np.int64), torch.int64)
        b.row_off, b.row_weight, b.E, b.delta_omega = (t.data_ptr() for t in (row_off, w, E, dom))
        for k in RECORD_FIELDS:
            setattr(b, k, rec[k].data_ptr())
        b.scale = 1.0
        b.sinc_cutoff = 0.0 if sinc_cutoff is None else float(sinc_cutoff)
        work, nbytes = _work(h, n_row, n_line, n_E, decoherence is not None)
        b.work, b.work_bytes = work.data_ptr(), nbytes
        a.base = b
        a.fields = fields.data_ptr()
        if decoherence is not None:
            a.elec_id, a.power = rec["elec_id"].data_ptr(), power.data_ptr()
        L.check(lib.pb_coherent_accumulate(C.byref(a), _stream_ptr(None)), "pb_coherent_accumulate")
    F = None
    if decoherence is not None:
        F = decoherence_factor(rows.G, decoherence["A_pop"], decoherence["xy0_pop"], decoherence["omega"],
                               device=dev)
    spec = h.zeros((n_E,), torch.float64)
    L.check(lib.pb_coherent_finalize(n_row, n_E, w.data_ptr(), fields.data_ptr(),
                                     power.data_ptr() if power is not None else None,
                                     F.data_ptr() if F is not None else None, 1.0 / int(segments["Ne"]),
                                     spec.data_ptr(), _stream_ptr(None)), "pb_coherent_finalize")
    return spec.cpu().numpy()


def decoherence_factor(G, A_pop, xy0_pop, omega, *, device=None, stream=None) -> torch.Tensor:
    """Row factors ``F[r, k] = |<exp(i (omega_k A_p - G_r,perp . xy0_p))>_p|^2``
    over the sampled population (``cxr/_per_hkl.py:121-160``,
    ``cxr/_setup.py:745-760``), FP64 on the device: [n_row, n_E]."""
    dev = _device(device)
    h = _Holder(dev)
    G = h.f64(G).reshape(-1, 3)
    A = h.f64(A_pop).reshape(-1)
    xy = h.f64(xy0_pop).reshape(-1, 2)
    om = h.f64(omega).reshape(-1)
    if int(xy.shape[0]) != int(A.numel()):
        raise ValueError("A_pop and xy0_pop must describe the same population")
    n_row, n_pop, n_E = int(G.shape[0]), int(A.numel()), int(om.numel())
    F = torch.empty((n_row, n_E), dtype=torch.float64, device=dev)
    a = L.PbDecoherenceArgs()
    a.n_row, a.n_pop, a.n_E = n_row, n_pop, n_E
    a.G, a.A_pop, a.xy0_pop, a.omega, a.F = (t.data_ptr() for t in (G, A, xy, om, F))
    L.check(L.load().pb_decoherence_factor(C.byref(a), _stream_ptr(stream)), "pb_decoherence_factor")
    if stream is not None:
        for t in h.keep:
            t.record_stream(stream)
    return F


def coherent_spectrum_decoherent(records, elec_id, row_count, row_weight, G, A_pop, xy0_pop, E_grid_eV,
                                 delta_omega, omega, Ne, *, sinc_cutoff=None, device=None) -> np.ndarray:
    """The coherent route with the sampled-bunch decoherence blend, per
    electron: every row's ``(1 - F) grouped + F flat`` weighted and summed
    over rows, divided by ``Ne`` (``cxr/_batched_finalize.py:163-243``).
    ``G`` holds the rows' reciprocal vectors, ``A_pop`` / ``xy0_pop`` the
    population's emission-time and transverse offsets (records offset-free,
    ``cxr/_setup.py:637-642``)."""
    if Ne < 1:
        raise ValueError("Ne must be >= 1")
    F = decoherence_factor(G, A_pop, xy0_pop, omega, device=device)
    spec = coherent_reduce(records, row_count, row_weight, E_grid_eV, delta_omega, scale=1.0 / Ne,
                           sinc_cutoff=sinc_cutoff, device=device, elec_id=elec_id, F_row=F)
    return spec.cpu().numpy()


def run_coherent_reduction_kernel(E_r, aw, phase_slope, g_phase, c_s_re, c_s_im, c_p_re, c_p_im, E_grid, *, out,
                                  mosaic_weight=1.0, L_esc=None, delta_omega=None, half_dL=None, apb=None,
                                  bma=None, q=None, sinc_cutoff=None, config=None):
    """One row's coherent intensity accumulated into ``out`` (the reference's
    signature, ``coherent_jit_kernel.py:716-766``).

    Without the in-medium pair the phase is the vacuum one; without the
    formation group each line is the real sinc ``sin(v)/v`` of
    ``v = aw (E - E_r)``, i.e. the formation factor with ``apb = 2``,
    ``bma = q = half_dL = 0``. ``config`` is accepted for signature
    compatibility; the launch shape is the library's. ``out`` is a float64
    device tensor.
    """
    del config
    if (L_esc is None) != (delta_omega is None):
        raise ValueError("L_esc and delta_omega must be given together")
    formation = (half_dL, apb, bma, q)
    use_formation = half_dL is not None
    if any((f is None) != (not use_formation) for f in formation):
        raise ValueError("half_dL, apb, bma and q must be given together")
    if use_formation and L_esc is None:
        raise ValueError("the formation factor needs L_esc and delta_omega")
    n = int(np.asarray(E_r).size) if not torch.is_tensor(E_r) else int(E_r.numel())
    n_E = int(np.asarray(E_grid).size) if not torch.is_tensor(E_grid) else int(E_grid.numel())
    if n_E == 0 or n == 0:
        return out
    zeros = np.zeros(n)
    if L_esc is None:
        L_esc, delta_omega = zeros, np.zeros(n_E)
    if not use_formation:
        half_dL, apb, bma, q = zeros, np.full(n, 2.0), zeros, zeros
    records = dict(E_vac=E_r, a_vac=aw, phase_slope=phase_slope, g_phase=g_phase, cs_re=c_s_re, cs_im=c_s_im,
                   cp_re=c_p_re, cp_im=c_p_im, L_esc=L_esc, half_dL=half_dL, apb=apb, bma=bma, q=q)
    coherent_reduce(records, [n], [float(mosaic_weight)], E_grid, delta_omega, sinc_cutoff=sinc_cutoff,
                    spec=out, device=out.device)
    return out


def assign_rows(row_count, world: int):
    """Rows to ranks, largest first onto the least loaded rank (lines x
    energies is the cost, the same on every rank for one row). Returns one
    ascending array of row indices per rank; deterministic."""
    row_count = np.asarray(row_count, dtype=np.int64)
    if world < 1:
        raise ValueError("world must be >= 1")
    load = np.zeros(world, dtype=np.int64)
    owner = np.empty(row_count.size, dtype=np.int64)
    for r in np.argsort(-row_count, kind="stable"):
        k = int(np.argmin(load))
        owner[r] = k
        load[k] += row_count[r]
    return [np.flatnonzero(owner == k) for k in range(world)]


def coherent_reduce_sharded(records, row_count, row_weight, E_grid_eV, delta_omega, *, scale=1.0, sinc_cutoff=None,
                            process_group=None, reduce_fn=None, device=None) -> torch.Tensor:
    """The coherent reduction with rows spread over the ranks of
    ``process_group``: rows add incoherently, so each rank reduces whole rows
    (a row's lines interfere and never split across ranks) and one all-reduce
    sums the FP64 spectra. Every rank passes the full record set and gets the
    full spectrum. ``reduce_fn`` (default ``coherent_reduce``) takes the same
    arguments for one rank's rows and returns a float64 tensor on the
    process group's device."""
    import torch.distributed as dist

    reduce_fn = reduce_fn or coherent_reduce
    world = dist.get_world_size(process_group) if process_group is not None or dist.is_initialized() else 1
    rank = dist.get_rank(process_group) if world > 1 else 0
    row_count = np.asarray(row_count, dtype=np.int64)
    off = np.concatenate([[0], np.cumsum(row_count)])
    rows = assign_rows(row_count, world)[rank]
    lines = np.concatenate([np.arange(off[r], off[r + 1]) for r in rows]) if rows.size else np.zeros(0, np.int64)
    sub = {k: (records[k][torch.as_tensor(lines, device=records[k].device)] if torch.is_tensor(records[k])
               else np.asarray(records[k])[lines]) for k in RECORD_FIELDS}
    w = np.asarray(row_weight, dtype=np.float64)
    kw = dict(scale=scale, sinc_cutoff=sinc_cutoff)
    if device is not None:
        kw["device"] = device
    if rows.size == 0:  # more ranks than rows: one empty row, so the rank still joins the collective
        counts, weights = np.zeros(1, np.int64), np.zeros(1)
    else:
        counts, weights = row_count[rows], w[rows]
    spec = reduce_fn(sub, counts, weights, E_grid_eV, delta_omega, **kw)
    if world > 1:
        dist.all_reduce(spec, op=dist.ReduceOp.SUM, group=process_group)
    return spec
