"""Drop-in for warp_fdtd/solver.py: fixed-input 3-D FDTD on the B200.

Same constructor, validation (ValueError messages), attributes and methods as
the reference `Solver` (solver.py:53-264).  What changes underneath:

* fused E+H kernels instead of two sweeps per step: on the slab-CPML path
  (the default when rows fit one TMA box) the time-blocked kernel advances two
  steps per launch inside run() (csrc/step_block.cu, `time_block`), else one
  fused step per launch (csrc/step_fz.cu, step_tma.cu, step_fused.cu); fields
  and CPML state ping-pong between two buffers, so `E`, `H` and `hprev` are
  views of the buffer the step counter's parity selects and no hprev copy is
  ever written;
* materials are stored as uint8 indices into an inverse-permittivity table
  when the grid has at most 256 distinct values (material="auto"), else as
  float32 per cell;
* detectors accumulate K-frequency DFTs in float64 (detectors.py);
* graphs are torch CUDA graphs of `graph_steps` steps.
All device memory is torch tensors; every kernel runs through the C ABI.
"""

import ctypes
import json
import time
from pathlib import Path

import numpy as np
import torch

from . import _lib
from . import kernels as k
from .schedule import X_WEIGHT, Y_WEIGHT, balanced_schedule, split_segment_schedule
from ._lib import ptr
from .bundle import read_bundle

C0 = 299792458.0


def pack_coefficients(coeff, shape):
    """solver.py:16-29: rank active planes per axis; pad six histories to the largest slab.

    Returns the (3, L, 4) table whose last column is the small exact integer
    plane rank, and the packed psi column count."""
    packed = np.zeros((*coeff.shape[:2], 4), np.float32)
    packed[..., :3] = coeff
    slab_sizes = []
    for axis, length in enumerate(shape):
        active = coeff[axis, :length, 0] != 0
        packed[axis, :length, 3] = np.maximum(np.cumsum(active) - 1, 0)
        slab_sizes.append(int(active.sum()) * (int(np.prod(shape)) // length))
    return packed, max(1, *slab_sizes)


def slab_ranks(packed, shape):
    """Ranks of the slab psi layout (the full-z pipeline's own layout).

    Per axis, each CPML side is one window running from its first to its last
    active cell (the low side holds the active cells in the lower half of the
    axis, the high side the rest); z windows are widened to whole groups of
    four cells so a group's four psi values are one aligned 16-byte vector.
    Every cell of a window, active or not, is numbered consecutively, windows
    one after the other, so a tile of rows inside a window has affine ranks.
    Returns the table with column 3 replaced and the three window lengths."""
    out = packed.copy()
    out[..., 3] = 0
    lengths = []
    for axis, length in enumerate(shape):
        act = np.flatnonzero(packed[axis, :length, 0] != 0)
        half = (length + 1) // 2
        wins = []
        for side in (act[act < half], act[act >= half]):
            if len(side):
                lo, hi = int(side[0]), int(side[-1])
                if axis == 2:
                    lo, hi = lo // 4 * 4, hi // 4 * 4 + 3
                wins.append([lo, hi])
        if len(wins) == 2 and wins[1][0] <= wins[0][1] + 1:
            wins = [[wins[0][0], wins[1][1]]]
        rank = 0
        for lo, hi in wins:
            idx = np.arange(lo, min(hi + 1, out.shape[1]))
            out[axis, idx, 3] = rank + idx - lo
            rank += hi - lo + 1
        lengths.append(rank)
    return out, lengths


def owned_array_bytes(solver):
    """solver.py:32-50: live owned device-tensor storage (deduplicated by pointer).

    Excludes allocator, graph and driver overhead; not a peak measurement."""
    seen = set()

    def size(value):
        if isinstance(value, torch.Tensor):
            if value.device.type != "cuda":
                return 0
            p = value.untyped_storage().data_ptr()
            if p in seen:
                return 0
            seen.add(p)
            return int(value.untyped_storage().nbytes())
        if isinstance(value, dict):
            return sum(size(v) for v in value.values())
        if isinstance(value, (list, tuple)):
            return sum(size(v) for v in value)
        return 0

    return size(vars(solver)) + sum(size(vars(m)) for m in solver.monitors)


def cpml_coefficients(meta, data, shape, field):
    """solver.py:105-123: coeff[axis, pos] = (a, b, 1/kappa), default (0, 1, 1)."""
    coeff = np.zeros((3, max(shape), 3), np.float32)
    coeff[:, :, 1:] = 1
    covered = np.zeros((3, max(shape)), bool)
    for obj in meta["objects"]:
        if obj["class"] != "PerfectlyMatchedLayer":
            continue
        name = obj["name"]
        dims = data[f"{name}/pml_a_{field}"].shape
        axis = int(np.argmax(dims))
        lo, hi = obj["grid_slice"][axis]
        if covered[axis, lo:hi].any():
            raise ValueError("Overlapping CPML slabs unsupported")
        covered[axis, lo:hi] = True
        for j, key in enumerate((f"pml_a_{field}", f"pml_b_{field}", f"inv_kappa_{field}")):
            coeff[axis, lo:hi, j] = data[f"{name}/{key}"].ravel()
    return coeff


def envelope(src, t):
    """Source envelope in float32.  SingleFrequencyProfile is the reference's
    ramp (solver.py:178-180); the two pulse profiles are this repository's
    extensions for broadband runs."""
    kind = src["temporal_profile"]
    if kind == "SingleFrequencyProfile":
        return np.clip(t / np.float32(src["num_startup_periods"] / src["frequency_hz"]), 0, 1)
    if kind == "GaussianPulseProfile":
        u = (t - np.float32(src["pulse_delay_s"])) / np.float32(src["pulse_sigma_s"])
        return np.exp(np.float32(-0.5) * u * u).astype(np.float32)
    if kind == "HannPulseProfile":
        u = (t - np.float32(src["pulse_delay_s"])) / np.float32(src["pulse_width_s"]) + np.float32(0.5)
        s = np.sin(np.float32(np.pi) * u)
        return np.where((u >= 0) & (u <= 1), s * s, np.float32(0)).astype(np.float32)
    raise ValueError(f"Unsupported temporal profile {kind}")


SUPPORTED_PROFILES = ("SingleFrequencyProfile", "GaussianPulseProfile", "HannPulseProfile")


class Solver:
    def __init__(self, case, device="cuda:0", graph_steps=64, cpml_storage="full",
                 material="auto", tile=None, path=0, schedule="balanced", time_block="auto"):
        if cpml_storage not in ("full", "packed"):
            raise ValueError("cpml_storage must be full or packed")
        if material not in ("auto", "u8", "f32"):
            raise ValueError("material must be auto, u8 or f32")
        self.cpml_storage = cpml_storage
        self.update_e = k.update_e_packed if cpml_storage == "packed" else k.update_e
        self.update_h = k.update_h_packed if cpml_storage == "packed" else k.update_h
        self.path = Path(case)
        self.meta, self.data = read_bundle(self.path)
        d, m = self.data, self.meta
        eps = d["inv_permittivity"]
        if eps.ndim != 4 or eps.shape[0] != 1 or not np.all(np.isfinite(eps)) or np.any(eps <= 0):
            raise ValueError("Only finite positive isotropic permittivity is supported")
        if d["inv_permeability"].ndim != 0 or d["inv_permeability"] != 1:
            raise ValueError("Only relative permeability 1 is supported")
        if m["settings"].get("precision", "float32") != "float32":
            raise ValueError("Only float32 field bundles supported")
        dx = m["settings"]["spacing_nm"] * 1e-9
        for axis in "xyz":
            if not np.allclose(np.diff(d[f"{axis}_edges_m"]), dx, rtol=1e-4, atol=0):
                raise ValueError("Only uniform cubic grids supported")
        self.shape = tuple(int(v) for v in eps.shape[1:])
        self.n = int(np.prod(self.shape))
        self.steps = int(m["time_steps"])
        if self.steps < 1 or not np.isfinite(m["dt_s"]) or m["dt_s"] <= 0:
            raise ValueError("Positive time step and trajectory length required")
        factor = m["settings"].get("courant_factor", 0.99)
        if not np.isfinite(factor) or not 0 < factor <= 0.99:
            raise ValueError("Require 0 < exported CFL factor <= 0.99")
        expected_dt = factor / np.sqrt(3) * dx / C0
        if not np.isclose(m["dt_s"], expected_dt, rtol=1e-4, atol=0):
            raise ValueError("Exported time step disagrees with the declared CFL factor")
        self.device = torch.device(device)
        if self.device.type != "cuda":
            raise ValueError("warp_fdtd_b200 runs on CUDA devices only")
        self.graph_steps = graph_steps
        if graph_steps < 1:
            raise ValueError("graph_steps must be positive")
        self.courant = factor / np.sqrt(3)
        self.tile = tuple(tile) if tile else (0, 0, 0)
        self.stages = 0
        if schedule not in ("balanced", "uniform"):
            raise ValueError("schedule must be balanced or uniform")
        # full-z path: cost-balanced one-wave block schedule, or uniform chunks
        # (also used whenever a tile sets chunk_x)
        self.schedule = schedule
        self.schedule_weights = (Y_WEIGHT, X_WEIGHT)
        if path not in (0, 1, 2, 3):
            raise ValueError("path must be 0 (auto), 1, 2 or 3")
        self.kernel_path = int(path)
        dev = self.device
        f32 = dict(dtype=torch.float32, device=dev)
        nx, ny, nz = self.shape
        # z rows padded to 16 B (fields, full psi, inv_eps) and 16 elements
        # (uint8 material) so the TMA pipeline can address every row; padding
        # cells stay zero and are never written.
        self._pitch = (nz + 3) // 4 * 4
        self._mpitch = (nz + 15) // 16 * 16
        self._cells = nx * ny * self._pitch
        self._E = [torch.zeros((3, self._cells), **f32) for _ in range(2)]
        self._H = [torch.zeros((3, self._cells), **f32) for _ in range(2)]
        self._issued = 0
        self.step = torch.zeros(1, dtype=torch.int32, device=dev)
        self._advance_counter = torch.zeros(1, dtype=torch.int32, device=dev)
        # status word of the step kernels: 0, or 1 (a bounded wait expired),
        # 2 (CPML ranks break the slab layout), 3 (bad schedule entry)
        self.kernel_status = torch.zeros(1, dtype=torch.int32, device=dev)

        # materials: uint8 index + table when possible, else float32 per cell
        flat = np.ascontiguousarray(eps.reshape(-1), np.float32)
        self.eps = torch.from_numpy(flat).to(dev)
        table, index = np.unique(flat, return_inverse=True)
        if material == "u8" and len(table) > 256:
            raise ValueError("material='u8' needs at most 256 distinct inverse permittivities")
        self.material = None
        self.material_table = None
        self._eps_p = None
        if material != "f32" and len(table) <= 256:
            self.material_kind = 1
            m8 = np.zeros((nx, ny, self._mpitch), np.uint8)
            m8[..., :nz] = index.astype(np.uint8).reshape(self.shape)
            self.material = torch.from_numpy(m8.reshape(-1)).to(dev)
            self.material_table = torch.from_numpy(table.astype(np.float32)).to(dev)
        else:
            self.material_kind = 0
            self._eps_p = torch.zeros(self._cells, **f32)
            self._sync_eps()

        # CPML tables (solver.py:105-131)
        self.coeffs, self._coeff4 = {}, {}
        tables = {f: cpml_coefficients(m, d, self.shape, f) for f in "EH"}
        packed = {f: pack_coefficients(tables[f], self.shape) for f in "EH"}
        for field in "EH":
            table = packed[field][0] if cpml_storage == "packed" else tables[field]
            self.coeffs[field] = torch.from_numpy(table).to(dev)
            self._coeff4[field] = torch.from_numpy(packed[field][0]).to(dev)
        # CPML state layout: the full-z pipeline (path 3, default when rows fit
        # one TMA box) keeps psi in slab blocks (x, y, z-rank); the other paths
        # use the reference's full or packed layout.
        use_slab = self.kernel_path in (0, 3) and self._pitch <= 248
        if self.kernel_path == 3 and not use_slab:
            raise ValueError("path 3 needs nz <= 248")
        active = [max(int((packed[f][0][axis, :self.shape[axis], 0] != 0).sum()) for f in "EH")
                  for axis in range(3)]
        self._psi_r = (active[0], active[1], (active[2] + 3) // 4 * 4)
        # the table the fused step reads: reference plane ranks, or slab ranks
        self._coeff_step = self._coeff4
        if use_slab:
            self._psi_layout = 2
            slab = {f: slab_ranks(packed[f][0], self.shape) for f in "EH"}
            self._coeff_step = {f: torch.from_numpy(slab[f][0]).to(dev) for f in "EH"}
            self._psi_r = tuple(max(slab["E"][1][a], slab["H"][1][a]) for a in range(3))
            rx, ry, rz = self._psi_r
            self._psi_cols = max(1, 2 * rx * ny * self._pitch + 2 * ry * nx * self._pitch
                                 + 2 * nx * ny * rz)
            shape = (self._psi_cols,)
        else:
            self._psi_layout = 1 if cpml_storage == "packed" else 0
            self._psi_cols = (max(packed["E"][1], packed["H"][1]) if cpml_storage == "packed"
                              else self._cells)
            shape = (6, self._psi_cols)
        for field in "EH":
            setattr(self, "_psi_" + field.lower(), [torch.zeros(shape, **f32) for _ in range(2)])

        # plane mode source (solver.py:132-182)
        sources = [o for o in m["objects"] if o["class"] == "ModePlaneSource"]
        if len(sources) != 1:
            raise ValueError("Exactly one exported plane mode source required")
        src = sources[0]
        if (
            src["direction"] != "+"
            or src["propagation_axis"] != 0
            or src["temporal_profile"] not in SUPPORTED_PROFILES
        ):
            raise ValueError("Only +x single-frequency source supported")
        self.source_x = src["grid_slice"][0][0]
        if src["grid_slice"] != [
            [self.source_x, self.source_x + 1],
            [0, self.shape[1]],
            [0, self.shape[2]],
        ]:
            raise ValueError("Source must span complete yz plane")
        self.sources, self.waves = {}, {}
        name = src["name"]
        if not np.array_equal(d[name + "/_time_step_to_on_idx"], np.arange(self.steps)):
            raise ValueError("Switched source schedules are not supported")
        if src["temporal_profile"] == "SingleFrequencyProfile" and src["num_startup_periods"] <= 0:
            raise ValueError("Source must have a positive startup ramp")
        for field in "EH":
            profile = d[f"{name}/_{field}"]
            if np.iscomplexobj(profile):
                raise ValueError("Complex source profiles unsupported")
            self.sources[field] = torch.from_numpy(
                np.ascontiguousarray(profile.reshape(3, -1), np.float32)).to(dev)
            offsets = d[f"{name}/_time_offset_{field}"].reshape(3, -1)
            if not np.all(offsets == offsets[:, :1]):
                raise ValueError("Spatially varying source delays unsupported")
            # float32 arithmetic with the separate multiply/divide of solver.py:165-181
            half_step = np.float32(0.5 if field == "E" else 0.0)
            t = (
                np.arange(self.steps, dtype=np.float32)[None, :] + half_step + offsets[:, :1]
            ) * np.float32(m["dt_s"])
            period = np.float32(1 / src["frequency_hz"])
            phase = (
                np.float32(2 * np.pi) * t / period
                + np.float32(src["phase_shift"])
                + np.float32(src["profile_phase_shift"])
            )
            wave = envelope(src, t) * np.cos(phase) * np.float32(src["static_amplitude_factor"])
            self.waves[field] = torch.from_numpy(np.ascontiguousarray(wave, np.float32)).to(dev)
        self.monitors = []
        self.save_h_from = self.steps
        self.graphs = {}
        self._args = self._step_args()
        # time-blocked kernel (fdtd_step_block): single steps at depth 1 and,
        # with time_block 2, pairs of steps in one launch inside run()
        if time_block not in ("auto", 0, 1, 2):
            raise ValueError("time_block must be 'auto', 0, 1 or 2")
        self.time_block = 0
        if self._psi_layout == 2 and time_block != 0:
            self.time_block = 2 if time_block == "auto" else int(time_block)
        # Physical buffer j of E, H and the CPML state is passed to the
        # kernels as pair entry j ^ _rel: a two-step launch moves the state
        # to the other buffer while the step parity stays, so it flips _rel.
        self._rel = 0
        self._final_flip = 0
        self._block = {}
        # launch shape of the time-blocked kernel per depth: (tile rows, TMA
        # stages), 0 = the library's pick
        self.block_shape = {1: (0, 0), 2: (0, 0)}
        self._mid = None
        self._extra2 = None
        if self.time_block:
            self._block_setup()

    # -- buffers selected by the number of issued steps --------------------
    def _compact(self, buf, rows):
        """(rows, n) view of a padded buffer (a copy when rows are padded)."""
        if self._pitch == self.shape[2]:
            return buf
        nx, ny, nz = self.shape
        return buf.view(rows, nx, ny, self._pitch)[..., :nz].reshape(rows, self.n)

    @property
    def E(self):
        return self._compact(self._E[(self._issued & 1) ^ self._rel], 3)

    @property
    def H(self):
        return self._compact(self._H[(self._issued & 1) ^ self._rel], 3)

    @property
    def hprev(self):
        """H(n-1/2) after the last issued step (zeros before the first)."""
        return self._compact(self._H[((self._issued + 1) & 1) ^ self._rel], 3)

    def _psi_reference(self, buf, field):
        """CPML state in the reference layout: (6, n) by cell for
        cpml_storage="full", (6, packed size) by plane rank for "packed"
        (solver.py:124-131).  Inactive entries are zero."""
        if self._psi_layout == 1:
            return buf
        if self._psi_layout == 0:
            return self._compact(buf, 6)
        nx, ny, nz = self.shape
        P = self._pitch
        rx, ry, rz = self._psi_r
        c4 = self._coeff_step[field].cpu()
        full = torch.zeros((6, nx, ny, nz), dtype=torch.float32, device=self.device)
        xb = buf[: 2 * rx * ny * P].view(2, rx, ny, P)
        yb = buf[2 * rx * ny * P: 2 * rx * ny * P + 2 * ry * nx * P].view(2, ry, nx, P)
        zb = buf[2 * rx * ny * P + 2 * ry * nx * P:][: 2 * nx * ny * rz].view(2, nx, ny, rz)
        for x in range(nx):
            if float(c4[0, x, 0]) != 0.0:
                r = int(c4[0, x, 3])
                full[0:2, x] = xb[:, r, :, :nz]
        for y in range(ny):
            if float(c4[1, y, 0]) != 0.0:
                r = int(c4[1, y, 3])
                full[2:4, :, y] = yb[:, r, :, :nz]
        for z in range(nz):
            if float(c4[2, z, 0]) != 0.0:
                r = int(c4[2, z, 3])
                full[4:6, :, :, z] = zb[:, :, :, r]
        full = full.reshape(6, self.n)
        if self.cpml_storage == "packed":
            from .kernels import pack_index

            return pack_index(full, self._coeff4[field], self.shape)
        return full

    @property
    def psi_e(self):
        return self._psi_reference(self._psi_e[(self._issued & 1) ^ self._rel], "E")

    @property
    def psi_h(self):
        return self._psi_reference(self._psi_h[(self._issued & 1) ^ self._rel], "H")

    def _sync_eps(self):
        """Copy `eps` (n,) into the padded float32 material the kernel reads."""
        nx, ny, nz = self.shape
        self._eps_p.view(nx, ny, self._pitch)[..., :nz].copy_(self.eps.view(nx, ny, nz))

    def _step_args(self):
        a = _lib.StepArgs()
        for j in range(2):
            a.E[j] = ptr(self._E[j])
            a.H[j] = ptr(self._H[j])
            a.psi_e[j] = ptr(self._psi_e[j])
            a.psi_h[j] = ptr(self._psi_h[j])
        a.psi_cols = self._psi_cols
        a.psi_rx, a.psi_ry, a.psi_rz = self._psi_r
        a.coeff_e = ptr(self._coeff_step["E"])
        a.coeff_h = ptr(self._coeff_step["H"])
        a.clen = int(self._coeff4["E"].shape[1])
        a.packed = int(self._psi_layout)
        a.material_kind = self.material_kind
        if self.material_kind == 0:
            a.inv_eps = ptr(self._eps_p)
        if self.material_kind == 1:
            a.material = ptr(self.material)
            a.material_table = ptr(self.material_table)
            a.material_count = int(self.material_table.numel())
        a.src_e = ptr(self.sources["E"])
        a.src_h = ptr(self.sources["H"])
        a.waves_e = ptr(self.waves["E"])
        a.waves_h = ptr(self.waves["H"])
        a.waves_cols = self.steps
        a.source_x = int(self.source_x)
        a.courant = float(self.courant)
        a.step = ptr(self.step)
        a.nx, a.ny, a.nz = self.shape
        a.pitch_z = self._pitch
        a.material_pitch = self._mpitch
        a.tile_y, a.tile_z, a.chunk_x = (int(v) for v in self.tile)
        a.stages = self.stages
        a.path = int(self.kernel_path)
        a.error = ptr(self.kernel_status)
        self._schedule = None
        if self._psi_layout == 2 and self.schedule == "balanced" and a.chunk_x <= 0:
            # one wave of cost-balanced (tile, x run) blocks, see schedule.py
            _lib.call("fdtd_step_defaults", ctypes.byref(a))  # the tile height
            ce = self._coeff_step["E"].cpu().numpy()
            ch = self._coeff_step["H"].cpu().numpy()
            slots, runs = None, None
            for _ in range(3):  # the run length sizes shared memory, hence occupancy
                blocks, sms = ctypes.c_int(0), ctypes.c_int(0)
                _lib.call("fdtd_step_occupancy", ctypes.byref(a), ctypes.byref(blocks),
                          ctypes.byref(sms))
                if blocks.value * sms.value == slots:
                    break
                slots = blocks.value * sms.value
                runs = balanced_schedule(self.shape, a.tile_y, ce, ch, slots,
                                         *self.schedule_weights)
                a.chunk_x = int((runs[:, 2] - runs[:, 1]).max())
            self._schedule = torch.from_numpy(runs).to(self.device)
            a.schedule = ptr(self._schedule)
            a.schedule_blocks = int(runs.shape[0])
        return a

    def autotune(self, tiles=None, stages=(3, 2), weights=None, repeats=20):
        """Pick the step's launch shape by timing it on this grid.

        With the time-blocked kernel (time_block 1 or 2) the candidates are
        (temporal depth, tile rows, TMA stages): each is timed over `repeats`
        launches with CUDA events after a warm-up, as milliseconds per time
        step (a depth-2 launch counts two), and the fastest is kept, depth
        included (time_block drops to 1 when single steps win).  Otherwise the
        single-step kernel's (tile rows, TMA stages, schedule cost weights) are
        tuned.  Candidates that do not fit (shared memory, threads) are
        skipped.  The solver is reset afterwards.  Returns the timings
        {candidate: ms per step}."""
        if self._psi_layout != 2:
            raise ValueError("autotune tunes the full-z path (path 0 or 3)")
        if self.time_block:
            return self._autotune_block(tiles, stages, repeats)
        a = self._step_args()
        _lib.call("fdtd_step_defaults", ctypes.byref(a))
        base = int(a.tile_y)
        tiles = tiles or sorted({max(1, base - 1), base, base + 1})
        weights = weights or [self.schedule_weights, (0.6, 0.5), (1.2, 1.0)]
        stream = torch.cuda.current_stream(self.device)
        saved = (self.tile, self.stages, self.schedule_weights)
        timings = {}
        for ty in tiles:
            for st in stages:
                for w in weights:
                    self.schedule_weights = tuple(w)
                    try:
                        self.set_tile(ty, 0, 0, st)
                        for _ in range(3):
                            _lib.call("fdtd_step_fused", self._args, stream.cuda_stream)
                    except (ValueError, _lib.FdtdError):
                        continue
                    e0 = torch.cuda.Event(enable_timing=True)
                    e1 = torch.cuda.Event(enable_timing=True)
                    e0.record(stream)
                    for _ in range(repeats):
                        _lib.call("fdtd_step_fused", self._args, stream.cuda_stream)
                    e1.record(stream)
                    e1.synchronize()
                    timings[(ty, st, tuple(w))] = e0.elapsed_time(e1) / repeats
        if timings:
            ty, st, w = min(timings, key=timings.get)
            self.schedule_weights = w
            self.set_tile(ty, 0, 0, st)
        else:
            self.tile, self.stages, self.schedule_weights = saved
            self.set_tile(self.tile[0], self.tile[1], self.tile[2], self.stages)
        self.reset()
        return timings

    def _autotune_block(self, tiles, stages, repeats):
        stream = torch.cuda.current_stream(self.device)
        depths = (1, 2) if self.time_block == 2 else (1,)
        saved = (self.time_block, dict(self.block_shape))
        timings = {}
        for depth in depths:
            self.time_block = max(depths)
            auto = self._block[depth]["plan"].tile_y
            cands = tiles or sorted({max(1, auto - 2), max(1, auto - 1), auto, auto + 1})
            for ty in cands:
                for st in stages:
                    try:
                        self.set_block_shape(depth, ty, st)
                    except (ValueError, _lib.FdtdError):
                        continue
                    info = self._block[depth]
                    extra = self._pair_extra() if depth == 2 else info["extra"]
                    if extra is None:
                        continue

                    def launch():
                        _lib.call("fdtd_step_block", ctypes.byref(info["args"][self._rel]),
                                  ctypes.byref(info["plan"]), ctypes.byref(extra),
                                  stream.cuda_stream)

                    for _ in range(3):
                        launch()
                    e0 = torch.cuda.Event(enable_timing=True)
                    e1 = torch.cuda.Event(enable_timing=True)
                    e0.record(stream)
                    for _ in range(repeats):
                        launch()
                    e1.record(stream)
                    e1.synchronize()
                    timings[(depth, ty, st)] = e0.elapsed_time(e1) / repeats / depth
            self.block_shape[depth] = saved[1][depth]
        if timings:
            best = min(timings, key=timings.get)
            for depth in depths:  # each depth keeps its own fastest shape
                own = {c: v for c, v in timings.items() if c[0] == depth}
                if own:
                    d, ty, st = min(own, key=own.get)
                    self.block_shape[depth] = (ty, st)
            self.time_block = best[0]
        else:
            self.time_block, self.block_shape = saved
        self._block_setup()
        self._extra2 = None
        self.graphs = {}
        self.reset()
        return timings

    def set_tile(self, tile_y, tile_z, chunk_x=0, stages=0):
        """Change the fused kernel's launch shape (tile rows, tile z cells,
        planes per block with 0 for the schedule, TMA ring stages with 0 for the
        default); captured graphs are dropped."""
        self.tile = (int(tile_y), int(tile_z), int(chunk_x))
        self.stages = int(stages)
        self._args = self._step_args()
        self.graphs = {}

    def set_block_shape(self, depth, tile_y=0, stages=0):
        """Launch shape of the time-blocked kernel at `depth` (1 or 2): tile
        rows and TMA stages, 0 for the library's pick; captured graphs are
        dropped."""
        if depth not in (1, 2) or not self.time_block or depth > self.time_block:
            raise ValueError("set_block_shape: depth not enabled by this solver's time_block")
        self.block_shape[depth] = (int(tile_y), int(stages))
        self._block_setup()
        self._extra2 = None
        self.graphs = {}


    def refresh_material(self):
        """Propagate an in-place change of `eps` to the copy the fused kernel reads."""
        if self.material_kind != 0:
            raise ValueError("refresh_material needs material='f32'")
        self._sync_eps()

    def reset(self):
        for group in (self._E, self._H, self._psi_e, self._psi_h):
            for a in group:
                a.zero_()
        self.step.zero_()
        self._issued = 0
        self._rel = 0
        for monitor in self.monitors:
            monitor.reset()
        torch.cuda.synchronize(self.device)

    # -- time-blocked kernel ------------------------------------------------
    def _block_setup(self):
        """Plans, schedules and argument pairs of the time-blocked kernel."""
        ce = self._coeff_step["E"].cpu().numpy()
        ch = self._coeff_step["H"].cpu().numpy()
        for depth in ((1, 2) if self.time_block == 2 else (1,)):
            base = self._step_args()
            base.schedule, base.schedule_blocks = None, 0
            base.tile_y, base.stages = (int(v) for v in self.block_shape[depth])
            base.chunk_x = 0
            plan = _lib.BlockPlan()
            _lib.call("fdtd_step_block_prepare", ctypes.byref(base), depth, ctypes.byref(plan))
            slots = max(1, plan.blocks_per_sm) * max(1, plan.sms)
            runs, segments, interior = split_segment_schedule(self.shape, plan.tile_y, depth,
                                                              ce, ch, slots)
            nblocks = runs.shape[0] // segments
            sched = torch.from_numpy(runs).to(self.device)
            base.tile_y = plan.tile_y
            base.schedule = ptr(sched)
            base.schedule_blocks = int(nblocks)
            real = runs[runs[:, 0] >= 0]
            base.chunk_x = int((real[:, 2] - real[:, 1]).max())
            pair = [base, self._swapped(base)]
            extra = _lib.BlockExtra()
            extra.segments = int(segments)
            extra.interior_blocks = int(interior)
            scratch = None
            if depth == 2:
                nbytes = int(plan.scratch_block_bytes) * int(nblocks)
                scratch = torch.empty(max(1, nbytes // 4), dtype=torch.float32, device=self.device)
                extra.scratch = ptr(scratch)
                extra.scratch_bytes = nbytes
            self._block[depth] = {"plan": plan, "schedule": sched, "args": pair,
                                  "extra": extra, "scratch": scratch}

    @staticmethod
    def _swapped(a):
        b = _lib.StepArgs()
        ctypes.pointer(b)[0] = a
        for name in ("E", "H", "psi_e", "psi_h"):
            pa, pb = getattr(a, name), getattr(b, name)
            pb[0], pb[1] = pa[1], pa[0]
        return b

    def _ord(self, bufs):
        """The (entry 0, entry 1) pointers of a physical buffer pair as the
        kernels' parity convention sees them now."""
        return ptr(bufs[self._rel]), ptr(bufs[self._rel ^ 1])

    def _pair_extra(self):
        """Depth-2 extras: scratch plus the snapshot boxes the detectors
        sample; None when the attached monitors cannot be fed from a
        snapshot (then run() advances one step per launch)."""
        key = tuple(id(m) for m in self.monitors)
        if self._extra2 is not None and self._extra2[0] == key:
            return self._extra2[1]
        boxes, ok = [], True
        nx, ny, nz = self.shape
        for m in self.monitors:
            if getattr(m, "shared", None) is not None:
                continue
            lo, shape = getattr(m, "lo", None), getattr(m, "shape", None)
            if lo is None or not hasattr(m, "exact") or type(m).__name__ != "Monitor":
                ok = False
                break
            e = 1 if m.exact else 0
            box = [max(lo[0] - e, 0), lo[0] + shape[0], max(lo[1] - e, 0), lo[1] + shape[1],
                   lo[2], min(lo[2] + shape[2] + e, nz)]
            boxes.append(box)
        extra = None
        if ok and len(boxes) <= _lib.SNAP_BOXES_MAX:
            info = self._block[2]
            extra = _lib.BlockExtra()
            extra.scratch = info["extra"].scratch
            extra.scratch_bytes = info["extra"].scratch_bytes
            extra.segments = info["extra"].segments
            extra.interior_blocks = info["extra"].interior_blocks
            if boxes:
                if self._mid is None:
                    f32 = dict(dtype=torch.float32, device=self.device)
                    self._mid = (torch.zeros((3, self._cells), **f32),
                                 torch.zeros((3, self._cells), **f32))
                extra.snap_e, extra.snap_h = ptr(self._mid[0]), ptr(self._mid[1])
                extra.nsnap = len(boxes)
                for b, box in enumerate(boxes):
                    for j, v in enumerate(box):
                        extra.snap_box[b][j] = int(v)
        self._extra2 = (key, extra)
        return extra

    def _step_kernel(self, stream):
        """One fused step of the current buffers (no detectors, no advance)."""
        if self.time_block:
            info = self._block[1]
            _lib.call("fdtd_step_block", ctypes.byref(info["args"][self._rel]),
                      ctypes.byref(info["plan"]), ctypes.byref(info["extra"]), stream)
        else:
            _lib.call("fdtd_step_fused", self._args, stream)

    def _record(self, E, H, stream):
        """Detectors of the step just computed (E, H: the (entry 0, entry 1)
        pointer pairs they read) and the counter advance."""
        planes, grouped = self._staged_planes()
        for monitor in self.monitors:
            if id(monitor) not in grouped:
                monitor.launch(self, E, H)
        if grouped:
            # every staged phasor plane in one launch, which also advances the
            # step counter after all of its blocks have read it
            nx, ny, nz = self.shape
            _lib.call("fdtd_record_stage_many", E[0], E[1], H[0], H[1], ptr(self.step), planes,
                      len(planes), nx, ny, nz, self._pitch, ptr(self._advance_counter), 1, stream)
        else:
            _lib.call("fdtd_advance", ptr(self.step), 1, stream)
        self._issued += 1
        self._folds()

    def _folds(self):
        """Fold the staged steps of every phasor monitor whose batch ends at
        the step just issued (or at the last step)."""
        for monitor in self.monitors:
            if monitor.is_phasor and (self._issued % monitor.batch == 0
                                      or self._issued == self.steps):
                monitor.fold(self, self._issued)

    def launch_step(self):
        """One step: fused E+H update, detectors, advance (solver.py:194-237)."""
        if self._issued >= self.steps and not torch.cuda.is_current_stream_capturing():
            raise ValueError("Trajectory complete; call reset() before stepping again")
        stream = _lib.stream_handle(self.device)
        self._step_kernel(stream)
        self._after_update(stream)
        self._record(self._ord(self._E), self._ord(self._H), stream)

    def _launch_pair(self, extra):
        """Two steps in one launch (depth 2), then the detectors of both: the
        first reads the snapshot of E(n+1), H(n+1/2), the second reads it as
        H(n-1/2)."""
        stream = _lib.stream_handle(self.device)
        info = self._block[2]
        _lib.call("fdtd_step_block", ctypes.byref(info["args"][self._rel]),
                  ctypes.byref(info["plan"]), ctypes.byref(extra), stream)
        s = self._issued & 1
        cur = s ^ self._rel  # physical buffer of the input state
        midE = ptr(self._mid[0]) if self._mid is not None else ptr(self._E[cur ^ 1])
        midH = ptr(self._mid[1]) if self._mid is not None else ptr(self._H[cur ^ 1])
        # step t (parity s) samples E[s^1], H[s^1] and H(n-1/2) = H[s]; step
        # t+1 (parity s^1) samples E[s], H[s] and H(n+1/2) = H[s^1]
        sets = []
        for src in (cur, cur ^ 1):
            E, H = [None, None], [None, None]
            E[s], E[s ^ 1] = ptr(self._E[src]), midE
            H[s], H[s ^ 1] = ptr(self._H[src]), midH
            sets.append((E, H))
        if self._pair_staging():
            # both steps' planes staged by one launch, which also advances the
            # counter by two; no fold falls between the two steps
            planes, _ = self._staged_planes()
            nx, ny, nz = self.shape
            fields = (ctypes.c_void_p * 8)(*(sets[0][0] + sets[0][1] + sets[1][0] + sets[1][1]))
            _lib.call("fdtd_record_stage_pair", fields, ptr(self.step), planes, len(planes),
                      nx, ny, nz, self._pitch, ptr(self._advance_counter), stream)
            for _ in range(2):
                self._issued += 1
                self._folds()
        else:
            for E, H in sets:
                self._record(E, H, stream)
        self._rel ^= 1

    def _pair_staging(self):
        """Whether a pair's detectors can run as one staging launch: every
        monitor records through the grouped staging (or shares a plane that
        does), and no plane folds between the pair's two steps."""
        planes, grouped = self._staged_planes()
        if planes is None:
            return False
        mid = self._issued + 1
        for m in self.monitors:
            if getattr(m, "shared", None) is not None:
                continue
            if id(m) not in grouped or m.batch % 2 or mid % m.batch == 0 or mid == self.steps:
                return False
        return True

    def _segment(self, length, final):
        """Issue `length` steps: pairs where the time-blocked kernel runs them,
        an even number of pairs unless `final` (the trajectory's last segment,
        which ends with a single step so that hprev is H(n-1/2))."""
        extra = self._pair_extra() if self.time_block == 2 else None
        n2 = 0
        if extra is not None:
            n2 = (length - 1) // 2 if final else 2 * (length // 4)
        for _ in range(n2):
            self._launch_pair(extra)
        for _ in range(length - 2 * n2):
            self.launch_step()
        return n2

    def _after_update(self, stream):
        """Hook between the fused update and the detectors (the step counter
        not yet advanced); the adjoint driver records its design-box history
        here when it keeps the whole trajectory."""

    def _staged_planes(self):
        """The staged phasor monitors that share one recording launch: two to
        eight planes (else none, and each monitor records itself)."""
        mons = [m for m in self.monitors if getattr(m, "is_phasor", False)
                and m.shared is None and getattr(m, "stage", None) is not None]
        key = tuple(id(m) for m in mons)
        if getattr(self, "_staged_key", None) != key:
            self._staged_key = key
            self._staged = (None, frozenset())
            if 2 <= len(mons) <= 8:
                planes = (_lib.StagePlane * len(mons))()
                for pl, m in zip(planes, mons):
                    pl.indices, pl.stage = ptr(m.indices), ptr(m.stage)
                    pl.nsteps, pl.T = int(m.indices.numel()), int(m.batch)
                    pl.x0, pl.y0, pl.z0 = (int(v) for v in m.lo)
                    pl.sx, pl.sy, pl.sz = (int(v) for v in m.shape)
                    pl.exact = int(m.exact)
                self._staged = (planes, frozenset(key))
        return self._staged

    def _graph_segments(self):
        """Graph segments of a whole trajectory: (key, length, start, final).

        A pair's detector launches are captured for the step parity at its
        start, so with an odd graph_steps the full graphs (which then start
        on both parities) are captured once per starting parity."""
        G, N = self.graph_steps, self.steps
        if self.time_block == 2:
            last = N % G or min(G, N)
            full = (N - last) // G
            segs = [(("full", c & 1), G, c * G, False) for c in range(min(full, 2 if G & 1 else 1))]
            return segs + [("final", last, N - last, True)]
        return [(length, length, 0 if length == G else N - length, False)
                for length in sorted({G, N % G} - {0}) if length <= N]

    def step_launches(self):
        """(two-step launches, one-step launches) of a whole trajectory run
        through the captured graphs."""
        if self.time_block != 2 or self._pair_extra() is None:
            return 0, self.steps
        G, N = self.graph_steps, self.steps
        last = N % G or min(G, N)
        full = (N - last) // G
        pairs = full * 2 * (G // 4) + (last - 1) // 2
        return pairs, N - 2 * pairs

    def _replays(self):
        """The captured graphs of a whole trajectory, in replay order."""
        G, N = self.graph_steps, self.steps
        if self.time_block == 2:
            last = N % G or min(G, N)
            return ([self.graphs[("full", (c * G) & 1)] for c in range((N - last) // G)]
                    + [self.graphs["final"]])
        out = [self.graphs[G]] * (N // G)
        if N % G:
            out.append(self.graphs[N % G])
        return out

    def compile(self):
        start = time.perf_counter()
        with torch.cuda.device(self.device):
            if self.time_block == 2:
                self._pair_extra()  # buffers are allocated before any capture
            self.launch_step()
            torch.cuda.synchronize(self.device)
            self.reset()
            self._final_flip = 0
            for key, length, offset, final in self._graph_segments():
                # capture at the step offset where the graph will be replayed so
                # the detectors' folds land on the right steps: full graphs start
                # on multiples of graph_steps, the last graph ends the trajectory
                self._issued = offset
                self._rel = 0
                for m in self.monitors:
                    m._folded = offset
                g = torch.cuda.CUDAGraph()
                with torch.cuda.graph(g, capture_error_mode="relaxed"):
                    n2 = self._segment(length, final) if self.time_block == 2 else 0
                    if self.time_block != 2:
                        for _ in range(length):
                            self.launch_step()
                if final:
                    self._final_flip = n2 & 1
                self._issued = 0
                self._rel = 0
                self.graphs[key] = g
            self.reset()
        return time.perf_counter() - start

    def run(self):
        with torch.cuda.device(self.device):
            if not self.graphs:
                self._segment(self.steps - self._issued, final=True)
            else:
                for g in self._replays():
                    g.replay()
                self._issued += self.steps
                self._rel ^= self._final_flip
                for m in self.monitors:
                    m._folded = self.steps
            torch.cuda.synchronize(self.device)

    def fields(self):
        return {
            name: arr.cpu().numpy().reshape(3, *self.shape)
            for name, arr in [("E", self.E), ("H", self.H)]
        }

    def set_fields(self, E=None, H=None):
        """Load (3, n) or (3, nx, ny, nz) fields into the current buffers."""
        nx, ny, nz = self.shape
        for arr, bufs in ((E, self._E), (H, self._H)):
            if arr is None:
                continue
            src = torch.as_tensor(np.asarray(arr, np.float32)).reshape(3, nx, ny, nz)
            dst = bufs[(self._issued & 1) ^ self._rel].view(3, nx, ny, self._pitch)
            dst[..., :nz].copy_(src.to(self.device))

    def summary(self):
        return json.dumps({"shape": self.shape, "steps": self.steps,
                           "material_kind": self.material_kind,
                           "cpml_storage": self.cpml_storage})
