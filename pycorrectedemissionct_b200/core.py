"""Device-resident core of the XRF path: batched fp / bp / maps / solver steps on torch CUDA tensors.

Everything here calls ``libcorrct_b200.so`` through the C ABI; torch only provides
device memory and the current CUDA stream.  Inputs must already be CUDA tensors;
there is no CPU path.
"""

from __future__ import annotations

import ctypes
import threading
from collections import OrderedDict

import numpy as np
import torch

from . import _lib, geometry

MAPS_DTYPES = {
    "float32": (torch.float32, _lib.CCT_DTYPE_F32),
    "bfloat16": (torch.bfloat16, _lib.CCT_DTYPE_BF16),
    # line-integral fields (S, A, 1 + D, n, n): L_in, then L_out per detector; channel c of a field
    # slice uses exp(-(L_in + s_c L_out)) (``XrfCore.set_channels``)
    "fields-float32": (torch.float32, _lib.CCT_DTYPE_FIELDS_F32),
}

BP_MODES = {"reference": _lib.CCT_BP_REFERENCE, "symmetric": _lib.CCT_BP_SYMMETRIC, "adjoint": _lib.CCT_BP_ADJOINT}

DEFAULT_MAPS_WORKSPACE = 256 << 20


def require_cuda(device=None) -> torch.device:
    """The CUDA device to run on; raises when CUDA is unavailable (no CPU fallback)."""
    if not torch.cuda.is_available():
        raise RuntimeError("corrct_b200 needs a CUDA device (B200, sm_100a); no CPU fallback exists")
    if device is None:
        return torch.device("cuda", torch.cuda.current_device())
    device = torch.device(device)
    if device.type != "cuda":
        raise ValueError(f"corrct_b200 runs on CUDA devices only, got {device}")
    return device


def stream_handle(device: torch.device) -> int:
    return torch.cuda.current_stream(device).cuda_stream


def _ptr(t: torch.Tensor | None) -> int | None:
    return None if t is None else t.data_ptr()


def _check_tensor(t: torch.Tensor, shape: tuple, dtype: torch.dtype, device: torch.device, name: str) -> None:
    if not isinstance(t, torch.Tensor) or t.device != device:
        raise ValueError(f"{name} must be a CUDA tensor on {device}")
    if tuple(t.shape) != tuple(shape):
        raise ValueError(f"{name} has shape {tuple(t.shape)}, expected {tuple(shape)}")
    if t.dtype != dtype:
        raise ValueError(f"{name} has dtype {t.dtype}, expected {dtype}")
    if not t.is_contiguous():
        raise ValueError(f"{name} must be contiguous")


def _maps_stride(maps: torch.Tensor | None) -> int:
    """Elements between consecutive slices' maps (0 = dense)."""
    if maps is None or maps.shape[0] <= 1 or maps.is_contiguous():
        return 0
    return int(maps.stride(0))


class XrfCore:
    """Geometry tables on the device plus batched projection entry points.

    Parameters
    ----------
    n : int
        Volume side (square) and detector width.
    angles_rot_rad : array-like
        Rotation angles (cast to float32 like the reference backend).
    n_det : int
        Fluorescence detectors (maps per angle).
    weights : (A, D) array or None
        ``w_det[d] * w_angle[a, d]`` applied by the attenuated fp and the symmetric bp.
    """

    def __init__(self, n: int, angles_rot_rad, n_det: int = 1, weights=None, device=None, variant: int = 0):
        self.device = require_cuda(device)
        self.variant = int(variant)
        self.n = int(n)
        self.n_det = int(n_det)
        self.angles_rad32, self.angles_deg32 = geometry.backend_angles(angles_rot_rad)
        self.n_angles = len(self.angles_rad32)
        self.fp_mat_np = geometry.fp_matrices(self.angles_deg32, self.n)
        self.trig_np = geometry.bp_trig(self.angles_deg32)
        self.fp_mat = torch.from_numpy(self.fp_mat_np).to(self.device)
        self.trig = torch.from_numpy(self.trig_np).to(self.device)
        # per-angle staged-box strides of the slice-grouped fp (speed only)
        self.box_strides = torch.from_numpy(geometry.fp_box_strides(self.fp_mat_np)).to(self.device)
        self.intensities_np = None
        self.line_scale = None
        self.psf = None
        self.n_channels = 0
        self.channel_scale = None
        self._base_weights = None
        self.set_weights(weights)

    def set_channels(self, scales) -> None:
        """Fluorescence channels read from line-integral fields: slice s of a batch is channel
        s % C of field slice s // C, with map exp(-(L_in + scales[c] * L_out)).  None clears."""
        if scales is None:
            self.n_channels, self.channel_scale = 0, None
            return
        sc = np.asarray(scales, dtype=np.float32).reshape(-1)
        if sc.size < 1:
            raise ValueError("at least one channel scale is required")
        self.n_channels = int(sc.size)
        self.channel_scale = torch.from_numpy(np.ascontiguousarray(sc)).to(self.device)

    def set_weights(self, weights) -> None:
        """Detector x angle weights ``w_det[d] * w_angle[a, d]`` (None = ones)."""
        self._base_weights = None if weights is None else np.asarray(weights, dtype=np.float64).reshape(self.n_angles, self.n_det)
        self._sync_weights()

    def set_intensities(self, intensities) -> None:
        """Projection intensities (A,) (corrct ``projectors.py:199-201``), None to clear."""
        if intensities is None:
            self.intensities_np = None
            self.line_scale = None
        else:
            i = np.asarray(intensities, dtype=np.float64).reshape(self.n_angles)
            self.intensities_np = i
            self.line_scale = torch.from_numpy(i.astype(np.float32)).to(self.device)
        self._sync_weights()

    def set_psf(self, psf) -> None:
        """Detector point-spread function (1-D kernel), None to clear."""
        if psf is None:
            self.psf = None
        else:
            k = np.asarray(psf, dtype=np.float32).reshape(-1)
            if not 1 <= len(k) <= 1024:
                raise ValueError("the PSF must have between 1 and 1024 taps")
            self.psf = torch.from_numpy(np.ascontiguousarray(k)).to(self.device)

    def _sync_weights(self) -> None:
        w = self._base_weights
        if self.intensities_np is not None:
            base = np.ones((self.n_angles, self.n_det)) if w is None else w
            w = base * self.intensities_np[:, None]
        if w is None:
            self.weights = None
            self.weights_np = None
        else:
            self.weights_np = w.astype(np.float32)
            self.weights = torch.from_numpy(np.ascontiguousarray(self.weights_np)).to(self.device)

    def angle_range(self, rng: slice) -> "XrfCore":
        """The same geometry restricted to a contiguous range of its angles; the device tables are
        views of this core's (no recomputation, no copies)."""
        sub = XrfCore.__new__(XrfCore)
        sub.device, sub.variant, sub.n, sub.n_det = self.device, self.variant, self.n, self.n_det
        sub.angles_rad32, sub.angles_deg32 = self.angles_rad32[rng], self.angles_deg32[rng]
        sub.n_angles = len(sub.angles_rad32)
        sub.fp_mat_np, sub.trig_np = self.fp_mat_np[rng], self.trig_np[rng]
        sub.fp_mat, sub.trig, sub.box_strides = self.fp_mat[rng], self.trig[rng], self.box_strides[rng]
        sub.intensities_np = None if self.intensities_np is None else self.intensities_np[rng]
        sub.line_scale = None if self.line_scale is None else self.line_scale[rng]
        sub.psf = self.psf
        sub.n_channels, sub.channel_scale = self.n_channels, self.channel_scale
        sub._base_weights = None if self._base_weights is None else self._base_weights[rng]
        sub.weights_np = None if self.weights_np is None else self.weights_np[rng]
        sub.weights = None if self.weights is None else self.weights[rng]
        return sub

    # ------------------------------------------------------------------ descriptors
    def desc(self, n_slices: int, maps_dtype: int = _lib.CCT_DTYPE_F32, angles: slice | None = None) -> _lib.XrfDesc:
        d = _lib.XrfDesc()
        d.n = self.n
        d.n_det = self.n_det
        d.n_slices = int(n_slices)
        d.maps_dtype = maps_dtype
        d.variant = self.variant
        if angles is None:
            d.n_angles = self.n_angles
            d.fp_matrix = self.fp_mat.data_ptr()
            d.bp_trig = self.trig.data_ptr()
            d.weights = _ptr(self.weights)
            d.line_scale = _ptr(self.line_scale)
            d.fp_box_strides = self.box_strides.data_ptr()
        else:
            a0, a1 = angles.start, angles.stop
            d.n_angles = a1 - a0
            d.fp_matrix = self.fp_mat[a0:a1].data_ptr()
            d.bp_trig = self.trig[a0:a1].data_ptr()
            d.weights = None if self.weights is None else self.weights[a0:a1].data_ptr()
            d.line_scale = None if self.line_scale is None else self.line_scale[a0:a1].data_ptr()
            d.fp_box_strides = self.box_strides[a0:a1].data_ptr()
        d.psf = _ptr(self.psf)
        d.psf_len = 0 if self.psf is None else int(self.psf.numel())
        if maps_dtype == _lib.CCT_DTYPE_FIELDS_F32:
            d.n_channels = self.n_channels
            d.channel_scale = _ptr(self.channel_scale)
        return d

    # ------------------------------------------------------------------ projections
    def fp(
        self,
        vol: torch.Tensor,
        maps: torch.Tensor | None = None,
        out: torch.Tensor | None = None,
        angles: slice | None = None,
    ) -> torch.Tensor:
        """Batched forward projection: vol (S, n, n) -> sino (S, D, A', n).

        ``angles`` (a contiguous slice) restricts the projection to those angles; ``maps``
        then holds only those angles: (S, A', D, n, n).
        """
        n = self.n
        s = vol.shape[0]
        na = self.n_angles if angles is None else angles.stop - angles.start
        _check_tensor(vol, (s, n, n), torch.float32, self.device, "vol")
        mdt = _lib.CCT_DTYPE_F32
        if maps is not None:
            mdt = self._check_maps(maps, s, na)
        elif self.n_det != 1:
            raise ValueError("an uncorrected projection needs a single detector")
        if out is None:
            out = torch.empty((s, self.n_det, na, n), dtype=torch.float32, device=self.device)
        _check_tensor(out, (s, self.n_det, na, n), torch.float32, self.device, "sino")
        desc = self.desc(s, mdt, angles)
        desc.maps_slice_stride = _maps_stride(maps)
        _lib.call("cct_fp", ctypes.byref(desc), vol.data_ptr(), _ptr(maps), out.data_ptr(), stream_handle(self.device))
        return out

    def bp(
        self,
        sino: torch.Tensor,
        mode: str = "reference",
        maps: torch.Tensor | None = None,
        out: torch.Tensor | None = None,
        angles: slice | None = None,
    ) -> torch.Tensor:
        """Batched back projection: sino (S, D, A', n) -> vol (S, n, n)."""
        n = self.n
        s = sino.shape[0]
        na = self.n_angles if angles is None else angles.stop - angles.start
        _check_tensor(sino, (s, self.n_det, na, n), torch.float32, self.device, "sino")
        if mode not in BP_MODES:
            raise ValueError(f"Unknown back-projection mode {mode!r}; expected one of {sorted(BP_MODES)}")
        mdt = _lib.CCT_DTYPE_F32
        if maps is not None:
            mdt = self._check_maps(maps, s, na)
        if out is None:
            out = torch.empty((s, n, n), dtype=torch.float32, device=self.device)
        _check_tensor(out, (s, n, n), torch.float32, self.device, "vol")
        desc = self.desc(s, mdt, angles)
        desc.maps_slice_stride = _maps_stride(maps)
        _lib.call(
            "cct_bp", ctypes.byref(desc), BP_MODES[mode], sino.data_ptr(), _ptr(maps), out.data_ptr(),
            stream_handle(self.device),
        )
        return out

    def _check_maps(self, maps: torch.Tensor, s: int, n_angles: int | None = None) -> int:
        """Maps (S, A', D, n, n): each slice's block contiguous; the slices may be further apart
        (an angle range of larger maps, ``maps[:, a0:a1]``)."""
        na = self.n_angles if n_angles is None else n_angles
        if self.n_channels > 0 and maps.dim() == 5 and maps.shape[2] == self.n_det + 1:
            # line-integral fields of s / C field slices
            if s % self.n_channels:
                raise ValueError(f"{s} slices are not a whole number of {self.n_channels}-channel field slices")
            fshape = (s // self.n_channels, na, self.n_det + 1, self.n, self.n)
            if maps.shape[0] > 1 and maps[0].is_contiguous() and maps.stride(0) >= maps[0].numel():
                _check_tensor(maps[0], fshape[1:], torch.float32, self.device, "fields")
                if tuple(maps.shape) != fshape:
                    raise ValueError(f"fields have shape {tuple(maps.shape)}, expected {fshape}")
            else:
                _check_tensor(maps, fshape, torch.float32, self.device, "fields")
            return _lib.CCT_DTYPE_FIELDS_F32
        shape = (s, na, self.n_det, self.n, self.n)
        dtype = torch.bfloat16 if maps.dtype == torch.bfloat16 else torch.float32
        if maps.dim() == 5 and maps.shape[0] > 1 and maps[0].is_contiguous() and maps.stride(0) >= maps[0].numel():
            _check_tensor(maps[0], shape[1:], dtype, self.device, "maps")
            if tuple(maps.shape) != shape:
                raise ValueError(f"maps has shape {tuple(maps.shape)}, expected {shape}")
        else:
            _check_tensor(maps, shape, dtype, self.device, "maps")
        return _lib.CCT_DTYPE_BF16 if dtype == torch.bfloat16 else _lib.CCT_DTYPE_F32

    def partials_count(self, n_slices: int) -> int:
        c = ctypes.c_int64(0)
        desc = self.desc(n_slices)
        _lib.call("cct_solver_partials_count", ctypes.byref(desc), ctypes.byref(c))
        return int(c.value)


_MAPS_TABLES: OrderedDict = OrderedDict()
_MAPS_TABLES_MAX = 16
_MAPS_TABLES_LOCK = threading.Lock()


def _maps_tables(device, n, angles_rad32, det_angles, surfaces_mm2, distances_mm, sub_sampling, half_turns):
    """Device rotation tables (and half-turn pairs) of one geometry, built on the host once and
    kept for the next calls with the same geometry (least recently used of 16 dropped)."""
    a32 = np.ascontiguousarray(np.array(angles_rad32, ndmin=1, dtype=np.float32))

    def key_of(v):
        return None if v is None else tuple(np.array(v, ndmin=1, dtype=np.float64).tolist())

    key = (str(device), int(n), a32.tobytes(), key_of(det_angles), key_of(surfaces_mm2), key_of(distances_mm),
           int(sub_sampling), bool(half_turns))
    with _MAPS_TABLES_LOCK:
        hit = _MAPS_TABLES.get(key)
        if hit is not None:
            _MAPS_TABLES.move_to_end(key)
            return hit
    rot_in, rot_out, n_sub = geometry.attenuation_rotations(a32, det_angles, n, surfaces_mm2, distances_mm, sub_sampling)
    rot_in_d = torch.from_numpy(np.ascontiguousarray(rot_in)).to(device)
    rot_out_d = torch.from_numpy(np.ascontiguousarray(rot_out)).to(device)
    pairs = geometry.half_turn_pairs(a32) if half_turns else None
    pairs_d = None if pairs is None else torch.from_numpy(pairs).to(device)
    quads = None
    if pairs is not None and n_sub == 1 and rot_out.shape[1] == 1:
        quads = geometry.quarter_turn_quads(a32, pairs, float(np.array(det_angles, ndmin=1, dtype=np.float64)[0]))
    quads_d = None if quads is None else torch.from_numpy(quads).to(device)
    entry = (rot_in_d, rot_out_d, n_sub, pairs_d, quads_d)
    with _MAPS_TABLES_LOCK:
        _MAPS_TABLES[key] = entry
        while len(_MAPS_TABLES) > _MAPS_TABLES_MAX:
            _MAPS_TABLES.popitem(last=False)
    return entry


def compute_maps(
    mu_in: torch.Tensor | None,
    mu_out: torch.Tensor | None,
    angles_rad32,
    det_angles=(np.pi / 2,),
    surfaces_mm2=None,
    distances_mm=None,
    sub_sampling: int = 1,
    maps_dtype: str = "float32",
    workspace: torch.Tensor | None = None,
    workspace_bytes: int = DEFAULT_MAPS_WORKSPACE,
    out: torch.Tensor | None = None,
    half_turns: bool = True,
    emitted_scale: float | None = None,
    quarter_turns: bool = True,
) -> torch.Tensor:
    """Attenuation maps (S, A, D, n, n) on the device from mu_in / mu_out (S, n, n) float32.

    ``half_turns``: angles whose half-turn partner (angle + pi) is also in the set share one
    rotation per direction (``geometry.half_turn_pairs``); False computes every angle on its own.
    ``emitted_scale``: the caller's statement that mu_out = emitted_scale * mu_in (taken as 1 when
    ``mu_out`` is ``mu_in`` itself).  With it, one point detector whose emitted direction is another
    angle's incident direction (``geometry.quarter_turn_quads``, e.g. a detector at pi / 2 and an
    angle count divisible by 4 over a full turn) and ``quarter_turns``, only incident fields are
    scanned: each angle's emitted line integral is emitted_scale times the incident one of the
    angle a quarter turn on.
    """
    ref = mu_in if mu_in is not None else mu_out
    if ref is None:
        raise ValueError("No attenuation volumes were given.")
    device = require_cuda(ref.device)
    s, n = ref.shape[0], ref.shape[-1]
    for name, t in (("mu_in", mu_in), ("mu_out", mu_out)):
        if t is not None:
            _check_tensor(t, (s, n, n), torch.float32, device, name)
    if maps_dtype not in MAPS_DTYPES:
        raise ValueError(f"maps_dtype must be one of {sorted(MAPS_DTYPES)}")
    tdt, cdt = MAPS_DTYPES[maps_dtype]
    rot_in_d, rot_out_d, n_sub, pairs_d, quads_d = _maps_tables(
        device, n, angles_rad32, det_angles, surfaces_mm2, distances_mm, sub_sampling, half_turns
    )
    if emitted_scale is None and mu_out is not None and mu_out is mu_in:
        emitted_scale = 1.0
    use_quads = (quarter_turns and quads_d is not None and emitted_scale is not None and mu_in is not None
                 and mu_out is not None and cdt != _lib.CCT_DTYPE_FIELDS_F32)
    n_ang, n_det = rot_out_d.shape[0], rot_out_d.shape[1]
    desc = _lib.MapsDesc()
    desc.n, desc.n_angles, desc.n_det, desc.n_slices = n, n_ang, n_det, s
    desc.n_sub, desc.maps_dtype = n_sub, cdt
    desc.has_in, desc.has_out = int(mu_in is not None), int(mu_out is not None)
    desc.rot_in, desc.rot_out = rot_in_d.data_ptr(), rot_out_d.data_ptr()
    entries = n_ang
    if pairs_d is not None:
        desc.pairs, desc.n_entries = pairs_d.data_ptr(), pairs_d.shape[0]
        entries = pairs_d.shape[0]
    if use_quads:
        desc.quads, desc.n_quads, desc.emitted_scale = quads_d.data_ptr(), quads_d.shape[0], float(emitted_scale)
        entries = quads_d.shape[0]  # a quad takes one entry's workspace (two incident fields)
    need = ctypes.c_size_t(0)
    _lib.call("cct_maps_workspace_size", ctypes.byref(desc), 1, ctypes.byref(need))
    if workspace is None:
        # at least 8 angles (of the whole batch) per pass, at most all of them
        nbytes = min(max(int(workspace_bytes), 8 * int(need.value)), int(need.value) * entries)
        workspace = torch.empty(nbytes, dtype=torch.uint8, device=device)
    planes = n_det + 1 if cdt == _lib.CCT_DTYPE_FIELDS_F32 else n_det
    if out is None:
        maps = torch.empty((s, n_ang, planes, n, n), dtype=tdt, device=device)
    else:
        _check_tensor(out, (s, n_ang, planes, n, n), tdt, device, "out")
        maps = out
    compute_maps.last_passes = -(-entries // max(1, (workspace.numel() * workspace.element_size()) // int(need.value)))
    _lib.call(
        "cct_compute_maps", ctypes.byref(desc), _ptr(mu_in), _ptr(mu_out), maps.data_ptr(), workspace.data_ptr(),
        workspace.numel() * workspace.element_size(), stream_handle(device),
    )
    # the cached tables may be dropped from the cache (and freed) by a later call while this
    # launch still reads them on this stream: tie their memory to the stream's pending work
    stream = torch.cuda.current_stream(device)
    for t in (rot_in_d, rot_out_d, pairs_d, quads_d):
        if t is not None:
            t.record_stream(stream)
    # torch's caching allocator reuses a workspace allocated here only for work queued later on
    # the same stream, so dropping it here is safe
    return maps


def maps_entry_bytes(n: int, n_slices: int, n_det: int = 1, n_sub: int = 1, has_in: bool = True,
                     has_out: bool = True) -> int:
    """Workspace bytes ``compute_maps`` needs per entry of a pass (one angle, or one half-turn pair
    of angles) for a batch of ``n_slices`` slices (``cct_maps_workspace_size``)."""
    desc = _lib.MapsDesc()
    desc.n, desc.n_angles, desc.n_det, desc.n_slices, desc.n_sub = int(n), 1, int(n_det), int(n_slices), int(n_sub)
    desc.has_in, desc.has_out = int(has_in), int(has_out)
    need = ctypes.c_size_t(0)
    _lib.call("cct_maps_workspace_size", ctypes.byref(desc), 1, ctypes.byref(need))
    return int(need.value)


def reduce_norm(v: torch.Tensor, ord: int = 2) -> torch.Tensor:
    """Per-slice FP64 norm sums of a (S, ...) float32 CUDA tensor: sum |v| (ord 1) or sum v^2 (ord 2)."""
    device = require_cuda(v.device)
    if v.dtype != torch.float32 or not v.is_contiguous():
        raise ValueError("reduce_norm needs a contiguous float32 tensor")
    s = v.shape[0]
    count = v.numel() // s
    out = torch.empty(s, dtype=torch.float64, device=device)
    partials = torch.empty(s * 1024, dtype=torch.float64, device=device)
    _lib.call("cct_reduce_norm", v.data_ptr(), count, s, ord, out.data_ptr(), partials.data_ptr(), stream_handle(device))
    return out
