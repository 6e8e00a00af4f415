"""Device-resident tensor API over the C ABI (include/mmnorm_b200.h).

All inputs are CUDA tensors; calls are asynchronous on the current torch stream.
PyTorch provides device memory and streams only -- every computation is one of the
library's sm_100a kernels, reached through ctypes.

    image, vote = backproject(x, y, z, antenna_locs, rx_offsets, meas, wavelength, slope)
    normals, mask = surface_normals(image, vote, filter_percent=0.05)
"""
from __future__ import annotations

import ctypes

import torch

from . import _lib

C = 2.99792458e8


def _vp(t):
    return ctypes.c_void_p(t.data_ptr()) if t is not None else ctypes.c_void_p(0)


def _stream(device):
    return ctypes.c_void_p(torch.cuda.current_stream(device).cuda_stream)


def _plain(t):
    """The tensor with torch's lazy conjugate / negative views materialised: the kernels
    read raw memory through data_ptr(), which ignores those flags."""
    return t.resolve_conj().resolve_neg() if isinstance(t, torch.Tensor) else t


def _need(t, name, dtype, device, shape=None):
    if not isinstance(t, torch.Tensor):
        raise TypeError("%s must be a torch.Tensor" % name)
    if t.is_conj() or t.is_neg():
        raise ValueError("%s is a lazy conjugate/negative view; pass t.resolve_conj()" % name)
    if t.device != device:
        raise ValueError("%s is on %s, expected %s" % (name, t.device, device))
    if t.dtype != dtype:
        raise TypeError("%s must be %s, got %s" % (name, dtype, t.dtype))
    if not t.is_contiguous():
        raise ValueError("%s must be contiguous" % name)
    if shape is not None and tuple(t.shape) != tuple(shape):
        raise ValueError("%s must have shape %s, got %s" % (name, shape, tuple(t.shape)))
    return t


def make_problem(x_locs, y_locs, z_locs, antenna_locs, rx_offsets, meas, wavelength, slope,
                 fft_spacing=0.0, is_ti_radar=False, pos_offsets=None):
    """Validated ``mmn_problem`` for device tensors (meas: complex64 [A, F])."""
    dev = meas.device
    if dev.type != "cuda":
        raise ValueError("mmnorm_b200 runs on CUDA tensors only (got %s)" % dev)
    f32 = torch.float32
    _need(x_locs, "x_locs", f32, dev)
    _need(y_locs, "y_locs", f32, dev)
    _need(z_locs, "z_locs", f32, dev)
    _need(meas, "meas", torch.complex64, dev)
    if meas.dim() != 2:
        raise ValueError("meas must be [num_antennas, num_samples]")
    A, F = meas.shape
    _need(antenna_locs, "antenna_locs", f32, dev, (A, 3))
    if rx_offsets.dim() != 2 or rx_offsets.shape[1] != 3:
        raise ValueError("rx_offsets must be [R, 3]")
    _need(rx_offsets, "rx_offsets", f32, dev)
    if pos_offsets is not None:
        _need(pos_offsets, "pos_offsets", f32, dev, (A, 3))
    p = _lib.MmnProblem()
    p.num_x, p.num_y, p.num_z = x_locs.numel(), y_locs.numel(), z_locs.numel()
    p.x_locs, p.y_locs, p.z_locs = x_locs.data_ptr(), y_locs.data_ptr(), z_locs.data_ptr()
    p.num_antennas = A
    p.num_rx = rx_offsets.shape[0]
    p.antenna_locs = antenna_locs.data_ptr() if A else 0
    p.rx_offsets = rx_offsets.data_ptr()
    p.pos_offsets = pos_offsets.data_ptr() if pos_offsets is not None else 0
    p.num_samples = F
    p.meas = meas.data_ptr() if A else 0
    p.wavelength = float(wavelength)
    p.slope = float(slope)
    p.fft_spacing = float(fft_spacing)
    p.is_ti_radar = int(bool(is_ti_radar))
    return p


def workspace_bytes(problem, mode="mixed"):
    n = _lib.load().mmn_workspace_bytes(ctypes.byref(problem), _lib.MODES[mode], 1)
    if n == 0:
        raise _lib.MmnError(_lib.MMN_ERR_INVALID_ARGUMENT, "mmn_workspace_bytes")
    return n


def plan_info(problem, mode="mixed"):
    vals = [ctypes.c_int32() for _ in range(5)]
    rc = _lib.load().mmn_plan_info(ctypes.byref(problem), _lib.MODES[mode],
                                   *[ctypes.byref(v) for v in vals])
    _lib.check(rc, "mmn_plan_info")
    keys = ("tiles", "splits", "antennas_per_stage", "threads", "voxels_per_thread")
    out = {k: v.value for k, v in zip(keys, vals)}
    n = ctypes.c_int32()
    _lib.check(_lib.load().mmn_plan_launches(ctypes.byref(problem), _lib.MODES[mode],
                                             ctypes.byref(n)), "mmn_plan_launches")
    out["launches"] = n.value  # kernels backproject launches for this problem
    return out


def backproject(x_locs, y_locs, z_locs, antenna_locs, rx_offsets, meas, wavelength, slope, *,
                mode="mixed", fft_spacing=0.0, is_ti_radar=False, pos_offsets=None,
                want_vote=True, workspace=None):
    """Fused backprojection + vote.

    Returns ``image`` complex64 [NX, NY, NZ] (raw sum over virtual antennas and samples,
    not normalised) and ``vote`` complex64 [3, NX, NY, NZ] (or None).
    ``mode``: 'mixed' (FP64 range/wrap + FP32 recurrence), 'plain' (FP32 sincos per
    sample), 'interp' (reference interpolated mode; ``meas`` holds range-FFT bins) or
    'nufft' (the mixed form's sum by an 8-tap gather from each antenna's 2x oversampled
    grid, ~1e-7 from 'mixed', O(8) instead of O(F) per voxel and antenna; F <= ~1500).
    """
    meas = _plain(meas)
    p = make_problem(x_locs, y_locs, z_locs, antenna_locs, rx_offsets, meas, wavelength,
                     slope, fft_spacing, is_ti_radar, pos_offsets)
    dev = meas.device
    nx, ny, nz = p.num_x, p.num_y, p.num_z
    V = nx * ny * nz
    image = torch.empty(V, dtype=torch.complex64, device=dev)
    vote = torch.empty((3, V), dtype=torch.complex64, device=dev) if want_vote else None
    lib = _lib.load()
    if mode == "nufft":
        nbytes = lib.mmn_backproject_nufft_workspace_bytes(ctypes.byref(p))
        if nbytes == 0:
            raise _lib.MmnError(_lib.MMN_ERR_TOO_LARGE, "mmn_backproject_nufft_workspace_bytes")
        if workspace is None or workspace.numel() < nbytes:
            workspace = torch.empty(nbytes, dtype=torch.uint8, device=dev)
        rc = lib.mmn_backproject_nufft(ctypes.byref(p), _vp(image), _vp(vote), _vp(workspace),
                                       workspace.numel(), _stream(dev))
        _lib.check(rc, "mmn_backproject_nufft")
        return image.view(nx, ny, nz), (vote.view(3, nx, ny, nz) if vote is not None else None)
    nbytes = workspace_bytes(p, mode)
    if workspace is None or workspace.numel() < nbytes:
        workspace = torch.empty(nbytes, dtype=torch.uint8, device=dev)
    rc = lib.mmn_backproject(ctypes.byref(p), _lib.MODES[mode], _vp(image), _vp(vote),
                             _vp(workspace), workspace.numel(), _stream(dev))
    _lib.check(rc, "mmn_backproject")
    return image.view(nx, ny, nz), (vote.view(3, nx, ny, nz) if vote is not None else None)


def surface_normals(image, vote, filter_percent=0.05, want_raw=False):
    """Unit normals float32 [..., 3] (NaN outside the mask), the bool mask, and
    optionally the raw (un-normalised) normal Re(conj(I) W)/|I|."""
    dev = image.device
    shape = tuple(image.shape)
    V = image.numel()
    img = _plain(image).reshape(V)
    w = _plain(vote).reshape(3, V)
    _need(img, "image", torch.complex64, dev)
    _need(w, "vote", torch.complex64, dev)
    normals = torch.empty((V, 3), dtype=torch.float32, device=dev)
    mask = torch.empty(V, dtype=torch.uint8, device=dev)
    raw = torch.empty((V, 3), dtype=torch.float32, device=dev) if want_raw else None
    lib = _lib.load()
    nbytes = lib.mmn_normals_workspace_bytes(V)
    ws = torch.empty(nbytes, dtype=torch.uint8, device=dev)
    rc = lib.mmn_normals(V, _vp(img), _vp(w), float(filter_percent), _vp(normals), _vp(mask),
                         _vp(raw), _vp(ws), nbytes, _stream(dev))
    _lib.check(rc, "mmn_normals")
    out = (normals.view(*shape, 3), mask.view(shape).bool())
    if want_raw:
        out = out + (raw.view(*shape, 3),)
    return out


def image_max_abs(image, out=None):
    """max |image| as a float32 device tensor of one element (``out`` if given)."""
    dev = image.device
    img = _need(_plain(image).reshape(-1), "image", torch.complex64, dev)
    if out is None:
        out = torch.empty(1, dtype=torch.float32, device=dev)
    _need(out, "out", torch.float32, dev, (1,))
    _lib.check(_lib.load().mmn_image_max_abs(img.numel(), _vp(img), _vp(out), _stream(dev)),
               "mmn_image_max_abs")
    return out


def surface_normals_from_max(image, vote, max_abs, filter_percent=0.05, want_raw=False):
    """surface_normals with the mask threshold taken from ``max_abs`` (float32 device
    tensor of one element, e.g. the all-reduced maximum over every slab of a grid)."""
    dev = image.device
    shape = tuple(image.shape)
    V = image.numel()
    img = _plain(image).reshape(V)
    w = _plain(vote).reshape(3, V)
    _need(img, "image", torch.complex64, dev)
    _need(w, "vote", torch.complex64, dev)
    _need(max_abs, "max_abs", torch.float32, dev, (1,))
    normals = torch.empty((V, 3), dtype=torch.float32, device=dev)
    mask = torch.empty(V, dtype=torch.uint8, device=dev)
    raw = torch.empty((V, 3), dtype=torch.float32, device=dev) if want_raw else None
    rc = _lib.load().mmn_normals_from_max(V, _vp(img), _vp(w), _vp(max_abs),
                                          float(filter_percent), _vp(normals), _vp(mask),
                                          _vp(raw), _stream(dev))
    _lib.check(rc, "mmn_normals_from_max")
    out = (normals.view(*shape, 3), mask.view(shape).bool())
    if want_raw:
        out = out + (raw.view(*shape, 3),)
    return out


def read_status(workspace):
    """Synchronise and return (and clear) the in-kernel status word of a workspace."""
    st = ctypes.c_int32(0)
    rc = _lib.load().mmn_read_status(_vp(workspace), ctypes.byref(st),
                                     _stream(workspace.device))
    _lib.check(rc, "mmn_read_status")
    return st.value


def variants(mode="mixed"):
    lib = _lib.load()
    m = _lib.MODES[mode]
    out = []
    for i in range(lib.mmn_num_variants(m)):
        t, nt = ctypes.c_int32(), ctypes.c_int32()
        _lib.check(lib.mmn_variant_info(m, i, ctypes.byref(t), ctypes.byref(nt)),
                   "mmn_variant_info")
        name = lib.mmn_variant_name(m, i)
        out.append({"index": i, "name": name.decode() if name else None,
                    "voxels_per_thread": t.value, "threads": nt.value})
    return out


def set_variant(mode, index):
    _lib.check(_lib.load().mmn_set_variant(_lib.MODES[mode], int(index)), "mmn_set_variant")


def current_variant(mode="mixed"):
    """Index (into ``variants(mode)``) of the process-wide variant ``backproject`` uses."""
    return int(_lib.load().mmn_get_variant(_lib.MODES[mode]))


POSITION_PASSES = {"interp": 0, "horner": 1}


def set_position_pass(form):
    """How the backward evaluates the position gradient's per-(voxel, antenna) sample sums:
    "interp" (default; interpolation from a 2x oversampled per-antenna spectrum, F <= ~1500)
    or "horner" (two FP32 Horner chains over all samples).  Process-wide."""
    _lib.check(_lib.load().mmn_set_position_pass(POSITION_PASSES[form]), "mmn_set_position_pass")


INTERP_FAST_FORMS = {"packed": 0, "scalar": 1}


def set_interp_fast_form(form):
    """Form of the fast interpolated passes: "packed" (default; two voxels per thread in
    packed FP32 instructions) or "scalar"."""
    _lib.check(_lib.load().mmn_set_interp_fast_form(INTERP_FAST_FORMS[form]),
               "mmn_set_interp_fast_form")


def set_measurement_pass(form):
    """How the backward evaluates the measurement gradient: "interp" (default; spread onto
    each antenna's 2x oversampled grid, then one transform per antenna; F <= ~1500) or
    "horner" (a sum over voxels for every sample).  Process-wide."""
    _lib.check(_lib.load().mmn_set_measurement_pass(POSITION_PASSES[form]),
               "mmn_set_measurement_pass")


def position_variants():
    """Launch shapes of the interpolation-form position pass, by index."""
    lib = _lib.load()
    return [lib.mmn_position_variant_name(i).decode()
            for i in range(lib.mmn_num_position_variants())]


def set_position_variant(index):
    _lib.check(_lib.load().mmn_set_position_variant(int(index)), "mmn_set_position_variant")


def current_position_variant():
    """Index (into ``position_variants()``) of the process-wide position-pass launch shape."""
    return int(_lib.load().mmn_get_position_variant())


def backproject_backward(x_locs, y_locs, z_locs, antenna_locs, rx_offsets, meas, wavelength,
                         slope, grad_image, grad_vote, *, is_ti_radar=False, pos_offsets=None,
                         want_meas=True, want_pos=True):
    """Adjoint of the mixed-precision ``backproject``: (grad_meas complex64 [A, F] or None,
    grad_pos float32 [A, 3] or None) for upstream dL/dI, dL/dW (torch convention)."""
    meas = _plain(meas)
    p = make_problem(x_locs, y_locs, z_locs, antenna_locs, rx_offsets, meas, wavelength, slope,
                     0.0, is_ti_radar, pos_offsets)
    dev = meas.device
    V = p.num_x * p.num_y * p.num_z
    gI = _plain(grad_image).reshape(V).contiguous() if grad_image is not None else None
    gW = _plain(grad_vote).reshape(3, V).contiguous() if grad_vote is not None else None
    if gI is None and gW is None:
        gI = torch.zeros(V, dtype=torch.complex64, device=dev)
    A, F = meas.shape
    gm = torch.empty((A, F), dtype=torch.complex64, device=dev) if want_meas else None
    gp = torch.empty((A, 3), dtype=torch.float32, device=dev) if want_pos else None
    lib = _lib.load()
    nbytes = lib.mmn_backward_workspace_bytes(ctypes.byref(p))
    if nbytes == 0:
        raise _lib.MmnError(_lib.MMN_ERR_INVALID_ARGUMENT, "mmn_backward_workspace_bytes")
    ws = torch.empty(nbytes, dtype=torch.uint8, device=dev)
    rc = lib.mmn_backproject_backward(ctypes.byref(p), _vp(gI), _vp(gW), _vp(gm), _vp(gp),
                                      _vp(ws), nbytes, _stream(dev))
    _lib.check(rc, "mmn_backproject_backward")
    return gm, gp


class BackprojectFunction(torch.autograd.Function):
    """Differentiable fused backprojection + vote (mixed precision).

    Inputs differentiated: ``meas`` (complex64 [A, F]) and ``pos_offsets`` (float32
    [A, 3], added to every TX and RX position: trajectory calibration).  The backward runs
    the library's adjoint kernels; phasors are recomputed, not stored."""

    @staticmethod
    def forward(ctx, meas, pos_offsets, x_locs, y_locs, z_locs, antenna_locs, rx_offsets,
                wavelength, slope, is_ti_radar, mode="mixed"):
        image, vote = backproject(x_locs, y_locs, z_locs, antenna_locs, rx_offsets, meas,
                                  wavelength, slope, mode=mode, is_ti_radar=is_ti_radar,
                                  pos_offsets=pos_offsets)
        ctx.save_for_backward(meas, pos_offsets, x_locs, y_locs, z_locs, antenna_locs,
                              rx_offsets)
        ctx.consts = (wavelength, slope, is_ti_radar)
        # an output the loss does not use arrives as None, not zeros: without a vote term
        # the passes skip the vote terms
        ctx.set_materialize_grads(False)
        return image, vote

    @staticmethod
    def backward(ctx, grad_image, grad_vote):
        meas, pos, x, y, z, ant, rxo = ctx.saved_tensors
        wavelength, slope, ti = ctx.consts
        if grad_image is None and grad_vote is None:
            return (None,) * 11
        gm, gp = backproject_backward(
            x, y, z, ant, rxo, meas, wavelength, slope,
            grad_image.contiguous() if grad_image is not None else None,
            grad_vote.contiguous() if grad_vote is not None else None,
            is_ti_radar=ti, pos_offsets=pos, want_meas=ctx.needs_input_grad[0],
            want_pos=ctx.needs_input_grad[1])
        return gm, gp, None, None, None, None, None, None, None, None, None


def backproject_differentiable(x_locs, y_locs, z_locs, antenna_locs, rx_offsets, meas,
                               wavelength, slope, pos_offsets=None, is_ti_radar=False,
                               mode="mixed"):
    """(image, vote) with autograd to ``meas`` and ``pos_offsets``.  ``mode``: "mixed" or
    "nufft" (the same sums by interpolation; the adjoint's interpolation-form
    measurement pass is its exact transpose)."""
    if mode not in ("mixed", "nufft"):
        raise ValueError("gradients are implemented for mode 'mixed' and 'nufft'")
    if pos_offsets is None:
        pos_offsets = torch.zeros_like(antenna_locs)
    return BackprojectFunction.apply(meas, pos_offsets, x_locs, y_locs, z_locs, antenna_locs,
                                     rx_offsets, float(wavelength), float(slope),
                                     bool(is_ti_radar), mode)


def normals_differentiable(image, vote, eps=1e-30):
    """Unit normals from (image, vote) in torch ops (differentiable), no mask:
    n = Re(conj(I) W)/|I| normalised (surface_normal_est.cu:138-144, image_processor.py:396)."""
    mag = image.abs().clamp_min(eps)
    raw = (image.conj().unsqueeze(0) * vote).real / mag.unsqueeze(0)
    return raw / raw.norm(dim=0, keepdim=True).clamp_min(eps)


class BatchPlan:
    """Many objects in one persistent launch (mmn_batch_* in the C ABI).

    ``objects``: sequence of dicts with CUDA tensors ``x_locs, y_locs, z_locs,
    antenna_locs, rx_offsets, meas`` and scalars ``wavelength, slope`` (optional
    ``is_ti_radar``, ``pos_offsets``).  ``run()`` computes every object's image and vote
    into ``self.images[o]`` (complex64 [NX,NY,NZ]) and ``self.votes[o]``
    (complex64 [3,NX,NY,NZ]); ``capture()`` records ``run()`` into a CUDA graph that
    ``replay()`` re-launches.  The input tensors must stay alive and unmoved."""

    def __init__(self, objects, items_per_slot=8, want_vote=True):
        lib = _lib.load()
        self.objects = [dict(ob, meas=_plain(ob["meas"])) for ob in objects]
        n = len(self.objects)
        dev = self.objects[0]["meas"].device
        self.device = dev
        probs = (_lib.MmnProblem * n)()
        self.images, self.votes, self._shapes = [], [], []
        for o, ob in enumerate(self.objects):
            probs[o] = make_problem(ob["x_locs"], ob["y_locs"], ob["z_locs"], ob["antenna_locs"],
                                    ob["rx_offsets"], ob["meas"], ob["wavelength"], ob["slope"],
                                    0.0, ob.get("is_ti_radar", False), ob.get("pos_offsets"))
            shape = (probs[o].num_x, probs[o].num_y, probs[o].num_z)
            V = shape[0] * shape[1] * shape[2]
            self._shapes.append(shape)
            self.images.append(torch.empty(V, dtype=torch.complex64, device=dev))
            self.votes.append(torch.empty((3, V), dtype=torch.complex64, device=dev)
                              if want_vote else None)
        img_ptrs = (ctypes.c_void_p * n)(*[t.data_ptr() for t in self.images])
        vote_ptrs = (ctypes.c_void_p * n)(*[t.data_ptr() if t is not None else 0
                                            for t in self.votes])
        handle = ctypes.c_void_p()
        nbytes = ctypes.c_size_t()
        rc = lib.mmn_batch_create(probs, n, _lib.MODE_MIXED, ctypes.cast(img_ptrs, ctypes.c_void_p),
                                  ctypes.cast(vote_ptrs, ctypes.c_void_p), int(items_per_slot),
                                  ctypes.byref(handle), ctypes.byref(nbytes))
        _lib.check(rc, "mmn_batch_create")
        self._probs = probs
        self._handle = handle
        self.workspace = torch.empty(max(256, nbytes.value), dtype=torch.uint8, device=dev)
        rc = lib.mmn_batch_upload(handle, _vp(self.workspace), self.workspace.numel(),
                                  _stream(dev))
        _lib.check(rc, "mmn_batch_upload")
        self.graph = None

    def info(self):
        vals = [ctypes.c_int32() for _ in range(4)]
        _lib.check(_lib.load().mmn_batch_info(self._handle, *[ctypes.byref(v) for v in vals]),
                   "mmn_batch_info")
        return dict(zip(("items", "ctas", "threads", "voxels_per_thread"), [v.value for v in vals]))

    def run(self):
        rc = _lib.load().mmn_batch_run(self._handle, _vp(self.workspace), _stream(self.device))
        _lib.check(rc, "mmn_batch_run")

    def capture(self):
        """Record run() into a CUDA graph (warm-up run on a side stream first)."""
        s = torch.cuda.Stream(self.device)
        s.wait_stream(torch.cuda.current_stream(self.device))
        with torch.cuda.stream(s):
            self.run()
        torch.cuda.current_stream(self.device).wait_stream(s)
        self.graph = torch.cuda.CUDAGraph()
        with torch.cuda.graph(self.graph):
            self.run()
        return self.graph

    def replay(self):
        if self.graph is None:
            self.capture()
        self.graph.replay()

    def results(self):
        out = []
        for img, vote, shape in zip(self.images, self.votes, self._shapes):
            out.append((img.view(*shape), vote.view(3, *shape) if vote is not None else None))
        return out

    def __del__(self):
        h = getattr(self, "_handle", None)
        if h is not None and h.value:
            try:
                _lib.load().mmn_batch_destroy(h)
            except Exception:
                pass
            self._handle = None
