"""Renderer: the reference's render API on top of libspectral.so.

Method names follow the Taichi kernels of main.py so that the reference's
application loop (main.py:1826-1840) ports line for line:

    r = Renderer(create_scene(), RenderConfig(), eems=..., cmf=cs.cmf)
    r.clear_pixel_space()
    total_samples, blocks = 0, 0
    while total_samples < r.config.samples_per_pixel:
        total_samples += 1
        r.cast_rays((total_samples - 1) % r.config.bands, blocks)
        if total_samples % r.config.bands == 0:
            blocks += 1
            r.average_and_reset_block(blocks)
            rgb = r.color_rays()

Device memory and streams come from PyTorch (the library itself allocates its
film and scene buffers and takes the current torch stream).  Nothing here
computes on the CPU: every render call is a CUDA launch through the C ABI.
"""
import ctypes
import dataclasses
from dataclasses import dataclass

import numpy as np

from . import _lib
from .scene import compile_scene


@dataclass
class RenderConfig:
    """Render constants of main.py:11-35 (reference defaults)."""
    width: int = 400                # RENDER_WIDTH = IMAGE_WIDTH // RESOLUTION_SCALE
    height: int = 400
    bands: int = 25                 # SPECTRAL_BANDS
    lambda_min: float = 10.0        # WAVELENGTH_MIN [nm]
    lambda_max: float = 1210.0      # WAVELENGTH_MAX [nm]
    max_path_length: int = 7        # MAX_PATH_LENGTH
    scatter_bounces: int = 5        # SCATTER_BOUNCES
    epsilon: float = 1e-4           # EPSILON
    escape: float = 1e2             # ESCAPE
    aspect_ratio: float = 1.0       # ASPECT_RATIO
    fov_scale: float = 1.0          # 1 = the reference camera (half-FOV atan(1/2))
    samples_per_pixel: int = 7000   # SAMPLES_PER_PIXEL
    exposure: float = 1.0           # EXPOSURE
    gamma: float = 2.0              # GAMMA
    image_width: int = 800          # IMAGE_WIDTH (display resolution of color_rays)
    image_height: int = 800
    seed: int = 0
    scene_id: int = 0
    kernel: str = "wavefront"       # "wavefront" or "mega" (plain single-scene megakernel)
    block_size: int = 0
    blocks_per_sm: int = 0
    sort_keys: int = 0
    trace_budget: int = 0
    traversal: str = "default"      # two-child nodes: "default" (if-if loop) or "speculative" (while-while)
    occupancy: int = 0              # megakernel: 0 = 5 blocks/SM (96 registers), 8 = 8 blocks/SM (64 registers)
    queue_capacity: int = 0         # wavefront path slots (0 = one per pixel); see ts_config
    loop_host: int = 0              # wavefront loop iterations launched by the host (profiling)
    defer_passes: bool = False      # cast_rays queues passes; runs of consecutive passes launch as bundles
    device: int = 0

    @property
    def wavelength_step(self):
        return (self.lambda_max - self.lambda_min) / (self.bands - 1) if self.bands > 1 else 0.0

    def wavelengths(self):
        return np.linspace(self.lambda_min, self.lambda_max, self.bands)

    def to_c(self):
        c = _lib.TsConfig()
        c.width, c.height, c.bands = self.width, self.height, self.bands
        c.lambda_min_nm, c.lambda_max_nm = self.lambda_min, self.lambda_max
        c.max_path_length, c.scatter_bounces = self.max_path_length, self.scatter_bounces
        c.epsilon, c.escape = self.epsilon, self.escape
        c.aspect_ratio, c.fov_scale = self.aspect_ratio, self.fov_scale
        c.seed, c.scene_id, c.device = self.seed & 0xFFFFFFFF, self.scene_id & 0xFFFFFFFF, self.device
        c.kernel = {"mega": _lib.KERNEL_MEGA, "wavefront": _lib.KERNEL_WAVEFRONT}[self.kernel]
        c.block_size, c.blocks_per_sm, c.sort_keys = self.block_size, self.blocks_per_sm, self.sort_keys
        c.trace_budget = self.trace_budget
        c.traversal = {"default": 0, "speculative": 1}[self.traversal]
        c.occupancy = self.occupancy
        c.queue_capacity = self.queue_capacity
        c.loop_host = self.loop_host
        return c


def fov_scale_for(vertical_fov_degrees):
    """fov_scale giving a vertical field of view (the reference's is 2*atan(1/2))."""
    return 2.0 * np.tan(np.radians(vertical_fov_degrees) / 2.0)


class _CudaArray:
    """Zero-copy view of a device buffer owned by the library context."""

    def __init__(self, ptr, shape, typestr):
        self.__cuda_array_interface__ = {"shape": tuple(shape), "typestr": typestr, "data": (int(ptr), False),
                                         "version": 3, "strides": None}


def _stream():
    import torch
    return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)


class Renderer:
    """One scene on one GPU (a libspectral context)."""

    def __init__(self, scene_dict, config=None, eems=None, cmf=None, bvh=None, bvh_params=None, exact=None,
                 cmf_scale=None):
        import torch
        if not torch.cuda.is_available():
            raise RuntimeError("spectral_b200.Renderer needs a CUDA device (there is no CPU fallback)")
        self.config = config or RenderConfig()
        self.lib = _lib.load()
        self._ctx = ctypes.c_void_p()
        _lib.check(self.lib.ts_create(ctypes.byref(self.config.to_c()), ctypes.byref(self._ctx)))
        self.device = torch.device("cuda", self.config.device)
        self._pending = []  # deferred (pass_idx, band) of cast_rays, oldest first
        self.total_samples = 0
        self.num_blocks_completed = 0
        self._cam = None
        self.compiled = None
        # the reference's normalisation: step / (sum_k cmf_y * step) (main.py:392-394, 1620)
        self.cmf_scale = cmf_scale
        self.setup_scene(scene_dict, eems=eems, cmf=cmf, bvh=bvh, bvh_params=bvh_params, exact=exact)

    def view(self, config=None, camera=None):
        """Another camera on this renderer's scene (ts_create_view): a Renderer with
        its own config (resolution, depth, seed, scene id, launch settings),
        camera and film that renders this scene without uploading it again.
        ``config`` keeps this renderer's bands and wavelength range; ``camera`` is
        a create_scene() camera dictionary (default: this renderer's camera).
        This renderer must stay open while the view is used."""
        import torch
        self.flush()
        cfg = config or dataclasses.replace(self.config)
        v = Renderer.__new__(Renderer)
        v.config = cfg
        v.lib = self.lib
        v._ctx = ctypes.c_void_p()
        _lib.check(self.lib.ts_create_view(self._ctx, ctypes.byref(cfg.to_c()), ctypes.byref(v._ctx)))
        v.device = torch.device("cuda", cfg.device)
        v._pending = []
        v.total_samples = 0
        v.num_blocks_completed = 0
        v._cam = self._cam
        v.compiled = self.compiled
        v.cmf_scale = self.cmf_scale
        v._owner = self
        if camera is not None:
            v.update_camera(camera["origin"], camera["lookat"], camera["up"])
        return v

    # ---------------------------------------------------------------- lifecycle
    def close(self):
        self._pending = []
        if self._ctx:
            self.lib.ts_destroy(self._ctx)
            self._ctx = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def _check(self, status):
        _lib.check(status, self._ctx)

    def flush(self):
        """Launch the passes that cast_rays deferred (``defer_passes``): one
        ts_render_passes launch for the run (a single pass: ts_render_pass), on
        the stream current now.  Every method that touches the film, the scene,
        the camera or the launch settings flushes first, so deferral changes no
        result, only how many launches render the passes."""
        p = getattr(self, "_pending", None)
        if not p:
            return
        self._pending = []
        # one launch holds at most 2^31 - 1 paths: very large frames launch the run in chunks
        per = max(1, (2 ** 31 - 1) // max(1, self.config.width * self.config.height))
        for k in range(0, len(p), per):
            first_pass, first_band = p[k]
            n = min(per, len(p) - k)
            if n == 1:
                self._check(self.lib.ts_render_pass(self._ctx, first_pass, first_band, _stream()))
            else:
                self._check(self.lib.ts_render_passes(self._ctx, first_pass, n, first_band, _stream()))

    def set_launch_config(self, kernel=None, traversal=None, block_size=None, blocks_per_sm=None, sort_keys=None,
                          trace_budget=None, occupancy=None, queue_capacity=None, loop_host=None):
        """Change launch settings without re-uploading the scene (images do not depend on them)."""
        self.flush()
        upd = {k: v for k, v in dict(kernel=kernel, traversal=traversal, block_size=block_size,
                                     blocks_per_sm=blocks_per_sm, sort_keys=sort_keys,
                                     trace_budget=trace_budget, occupancy=occupancy,
                                     queue_capacity=queue_capacity, loop_host=loop_host).items()
               if v is not None}
        cfg = dataclasses.replace(self.config, **upd)
        self._check(self.lib.ts_set_launch_config(self._ctx, ctypes.byref(cfg.to_c())))
        self.config = cfg

    # ---------------------------------------------------------------- scene
    def setup_scene(self, scene_dict, eems=None, cmf=None, bvh=None, bvh_params=None, exact=None):
        """setup_scene + build_bvh (main.py:437-631): flatten, build the BVH, upload."""
        self.flush()
        cs = compile_scene(scene_dict, self.config.bands, eems=eems, cmf=cmf, bvh=bvh, bvh_params=bvh_params,
                           exact=exact)
        d = cs.desc()
        self._check(self.lib.ts_upload_scene(self._ctx, ctypes.byref(d)))
        self.compiled = cs
        if self.cmf_scale is None:
            ysum = float(np.sum(cs.cmf.astype(np.float64)[:, 1])) * self.config.wavelength_step
            self.cmf_scale = self.config.wavelength_step / ysum if ysum > 0 else 0.0
        cam = scene_dict.get("camera")
        if cam is not None:
            self.update_camera(cam["origin"], cam["lookat"], cam["up"])

    def scene_info(self):
        info = _lib.TsSceneInfo()
        self._check(self.lib.ts_scene_info_get(self._ctx, ctypes.byref(info)))
        return {k: getattr(info, k) for k, _ in info._fields_}

    def tri_perm(self):
        """slot -> original triangle index of the uploaded BVH order."""
        n = self.compiled.num_tris
        out = np.zeros(n, np.int32)
        self._check(self.lib.ts_get_tri_perm(self._ctx, out.ctypes.data_as(_lib.I32P)))
        return out

    # ---------------------------------------------------------------- camera
    def update_camera(self, origin=None, lookat=None, up=None):
        """update_camera (main.py:633-640); arguments replace the stored ones."""
        self.flush()
        o, l, u = self._cam or ([0.0, 0.0, 3.5], [0.0, 0.0, -1.0], [0.0, 1.0, 0.0])
        o = o if origin is None else origin
        l = l if lookat is None else lookat
        u = u if up is None else up
        self._cam = (list(map(float, o)), list(map(float, l)), list(map(float, u)))
        arr = lambda v: (ctypes.c_float * 3)(*v)
        self._check(self.lib.ts_set_camera(self._ctx, arr(self._cam[0]), arr(self._cam[1]), arr(self._cam[2])))

    # ---------------------------------------------------------------- render
    def cast_rays(self, current_sample_in_block, block_index=0, pass_idx=None):
        """One sample pass at band ``current_sample_in_block`` (main.py:1502-1590).

        pass_idx picks the random stream; by default it is the number of passes
        rendered since the last clear, so a cleared renderer replays the same
        sample sequence (common random numbers).

        With ``config.defer_passes`` the pass is queued instead: passes that
        continue the queued run (next pass index, next band mod B) join it, and
        the run is launched as one wavelength bundle when it holds B passes or
        when anything else needs the film (``flush``).  The reference's cadence
        -- B cast_rays, then average_and_reset_block -- then costs one launch
        per block."""
        if pass_idx is None:
            pass_idx = self.total_samples
        pass_idx = int(pass_idx) & 0xFFFFFFFF
        band = int(current_sample_in_block)
        B = self.config.bands
        if self.config.defer_passes and 0 <= band < B:
            p = self._pending
            if p and not (len(p) < B and pass_idx == (p[-1][0] + 1) & 0xFFFFFFFF and band == (p[-1][1] + 1) % B):
                self.flush()
            self._pending.append((pass_idx, band))
            if len(self._pending) == B:
                self.flush()
        else:
            self.flush()
            self._check(self.lib.ts_render_pass(self._ctx, pass_idx, band, _stream()))
        self.total_samples += 1

    def cast_rays_bundle(self, first_band, num_passes, pass_idx=None):
        """num_passes consecutive passes (bands first_band, first_band + 1, ... mod B) in one
        launch: the same paths as num_passes cast_rays calls (num_passes <= bands)."""
        self.flush()
        if pass_idx is None:
            pass_idx = self.total_samples
        self._check(self.lib.ts_render_passes(self._ctx, int(pass_idx) & 0xFFFFFFFF, int(num_passes),
                                              int(first_band), _stream()))
        self.total_samples += int(num_passes)

    def wave_loop_iterations(self):
        """Iterations (trace + shade + control launches) of the last regenerating wavefront launch."""
        self.flush()
        n = ctypes.c_int32(0)
        self._check(self.lib.ts_wave_loop_iterations(self._ctx, _stream(), ctypes.byref(n)))
        return int(n.value)

    def record_paths(self, first_pass=0, num_passes=0):
        """Arm path records for passes first_pass .. first_pass + num_passes - 1
        (0 disarms): renders of those passes run the megakernel and record each
        path's total deposit, which a later adjoint of the same passes uses in
        place of its weight replay."""
        self.flush()
        self._check(self.lib.ts_record_paths(self._ctx, int(first_pass) & 0xFFFFFFFF, int(num_passes)))

    def set_loop_iteration_limit(self, limit=0):
        """Bound on the iterations of one regenerating-loop launch (0 = automatic);
        a launch that reaches it stops on the device and check_device reports it."""
        self.flush()
        self._check(self.lib.ts_set_loop_iteration_limit(self._ctx, int(limit)))

    def cast_rays_counted(self, current_sample_in_block, pass_idx=None):
        """cast_rays through the counting megakernel; returns the work counts."""
        self.flush()
        if pass_idx is None:
            pass_idx = self.total_samples
        w = (ctypes.c_uint64 * 8)()
        self._check(self.lib.ts_render_pass_counted(self._ctx, int(pass_idx) & 0xFFFFFFFF,
                                                    int(current_sample_in_block), _stream(), w))
        self.total_samples += 1
        keys = ("paths", "vertices", "traces", "node_visits", "tri_tests", "hits", "deposits")
        return {k: int(w[i]) for i, k in enumerate(keys)}

    def average_and_reset_block(self, num_blocks_completed):
        """main.py:1592-1607 (FP64 running mean plus the per-cell sum of squares)."""
        self.flush()
        self._check(self.lib.ts_accumulate_block(self._ctx, int(num_blocks_completed), _stream()))
        self.num_blocks_completed = int(num_blocks_completed)

    def clear_pixel_space(self):
        """main.py:1661-1674."""
        self.flush()
        self._check(self.lib.ts_reset(self._ctx, _stream()))
        self.total_samples = 0
        self.num_blocks_completed = 0

    def render(self, samples=None, callback=None, bundles=True):
        """The pass/block cadence of main.py:1826-1837 for ``samples`` passes:
        pass k at band k mod B, the block averaged after every B passes (then
        ``callback(self)``).  bundles: each whole block is one launch
        (ts_render_passes: the same paths and deposits as B cast_rays calls)."""
        samples = self.config.samples_per_pixel if samples is None else samples
        B = self.config.bands
        left = int(samples)
        while left > 0:
            if bundles and left >= B and self.total_samples % B == 0:
                self.cast_rays_bundle(0, B)
                left -= B
            else:
                self.cast_rays(self.total_samples % B, self.num_blocks_completed)
                left -= 1
            if self.total_samples % B == 0:
                self.average_and_reset_block(self.num_blocks_completed + 1)
                if callback is not None:
                    callback(self)
        return self

    # ---------------------------------------------------------------- film views
    def _film(self, which):
        import torch
        self.flush()
        ptr = ctypes.POINTER(ctypes.c_double)()
        n = ctypes.c_size_t()
        self._check(self.lib.ts_film_buffer(self._ctx, which, ctypes.byref(ptr), ctypes.byref(n)))
        c = self.config
        addr = ctypes.cast(ptr, ctypes.c_void_p).value
        return torch.as_tensor(_CudaArray(addr, (c.bands, c.height, c.width), "<f8"), device=self.device)

    @property
    def block_film(self):
        """Current block's per-band sums, [B][H][W] float64 (device view)."""
        return self._film(_lib.FILM_BLOCK)

    @property
    def mean_film(self):
        """Running mean over completed blocks, [B][H][W] float64 (device view)."""
        return self._film(_lib.FILM_MEAN)

    @property
    def m2_film(self):
        """Sum over blocks of the squared block values, [B][H][W] float64 (device view)."""
        return self._film(_lib.FILM_M2)

    @property
    def spectral_accumulator(self):
        """The reference's spectral_accumulator[i, j, k] layout (a [W][H][B] view)."""
        return self.mean_film.permute(2, 1, 0)

    @property
    def block_accumulator(self):
        return self.block_film.permute(2, 1, 0)

    def standard_error(self):
        """Per-cell standard error of the block mean, [B][H][W] float64."""
        n = self.num_blocks_completed
        if n < 2:
            raise ValueError("need at least two completed blocks")
        mean, m2 = self.mean_film, self.m2_film
        var = (m2 / n - mean * mean).clamp_min(0.0) * (n / (n - 1))
        return (var / n).sqrt()

    # ---------------------------------------------------------------- resolve
    def resolve_xyz(self, out=None):
        """XYZ at render resolution, [H][W][3] float32 (XYZ half of color_rays)."""
        import torch
        self.flush()
        c = self.config
        if out is None:
            out = torch.empty((c.height, c.width, 3), dtype=torch.float32, device=self.device)
        self._check(self.lib.ts_resolve_xyz(self._ctx, float(self.cmf_scale), ctypes.c_void_p(out.data_ptr()),
                                            _stream()))
        return out

    def resolve_xyz_host(self, out=None):
        """Same, into a (pinned) host array; the stream is synchronised."""
        self.flush()
        c = self.config
        if out is None:
            out = np.empty((c.height, c.width, 3), np.float32)
        self._check(self.lib.ts_resolve_xyz_host(self._ctx, float(self.cmf_scale),
                                                 out.ctypes.data_as(_lib.F32P), _stream()))
        return out

    def color_rays(self, xyz_to_rgb=None, out=None):
        """color_rays (main.py:1609-1629): [image_height][image_width][3] float32 device image."""
        import torch
        self.flush()
        c = self.config
        if xyz_to_rgb is None:
            from .spectral_data import srgb_xyz_to_rgb
            xyz_to_rgb = srgb_xyz_to_rgb()
        m = (ctypes.c_float * 9)(*np.asarray(xyz_to_rgb, np.float64).reshape(9).tolist())
        if out is None:
            out = torch.empty((c.image_height, c.image_width, 3), dtype=torch.float32, device=self.device)
        self._check(self.lib.ts_resolve_rgb(self._ctx, float(self.cmf_scale), m, c.exposure, c.gamma,
                                            c.image_width, c.image_height, ctypes.c_void_p(out.data_ptr()),
                                            _stream()))
        return out

    def visualize_normals(self, out=None):
        """Geometry mode (main.py:1631-1659): shading normal * 0.5 + 0.5, [H][W][3]."""
        import torch
        c = self.config
        if out is None:
            out = torch.empty((c.height, c.width, 3), dtype=torch.float32, device=self.device)
        self._check(self.lib.ts_render_normals(self._ctx, ctypes.c_void_p(out.data_ptr()), _stream()))
        return out

    # ---------------------------------------------------------------- queries
    def trace(self, rays, mode="fast"):
        """Closest hit of [n][6] rays (a torch CUDA tensor) -> (tri, t, u, v).

        tri is the ORIGINAL triangle index (-1 on a miss), t = 1e9 on a miss.
        mode "reference_order" walks the tree exactly like the reference's trace.
        """
        import torch
        rays = rays.to(device=self.device, dtype=torch.float32).contiguous()
        n = rays.shape[0]
        tri = torch.empty(n, dtype=torch.int32, device=self.device)
        t = torch.empty(n, dtype=torch.float32, device=self.device)
        u = torch.empty(n, dtype=torch.float32, device=self.device)
        v = torch.empty(n, dtype=torch.float32, device=self.device)
        m = {"fast": _lib.TRACE_FAST, "reference_order": _lib.TRACE_REFERENCE_ORDER}[mode]
        p = lambda x: ctypes.c_void_p(x.data_ptr())
        self._check(self.lib.ts_trace_batch(self._ctx, p(rays), n, m, p(tri), p(t), p(u), p(v), _stream()))
        return tri, t, u, v

    # ---------------------------------------------------------------- differentiation
    def param_count(self):
        """(material-table entries M*6*B, EEM entries E*B*B) of the parameter vector."""
        a, b = ctypes.c_int64(), ctypes.c_int64()
        self._check(self.lib.ts_param_count(self._ctx, ctypes.byref(a), ctypes.byref(b)))
        return a.value, b.value

    def update_materials(self, mat_f32=None, eem=None):
        """Replace the material table [M,6,B] and/or EEM table [E,B,B] (float32 CUDA tensors)."""
        import torch
        self.flush()
        p = lambda x: None if x is None else ctypes.c_void_p(x.data_ptr())
        keep = []
        for x in (mat_f32, eem):
            if x is not None:
                if x.device != self.device or x.dtype != torch.float32 or not x.is_contiguous():
                    raise ValueError("update_materials expects contiguous float32 tensors on the renderer's device")
                keep.append(x)
        M, E = self.compiled.mat_f32.shape[0], self.compiled.eem.shape[0]
        B = self.config.bands
        if mat_f32 is not None and tuple(mat_f32.shape) != (M, 6, B):
            raise ValueError(f"mat_f32 must be [{M}, 6, {B}]")
        if eem is not None and tuple(eem.shape) != (E, B, B):
            raise ValueError(f"eem must be [{E}, {B}, {B}]")
        self._check(self.lib.ts_update_materials(self._ctx, p(mat_f32), p(eem), _stream()))
        self.materials_version = getattr(self, "materials_version", 0) + 1

    def adjoint_pass(self, current_sample_in_block, pass_idx, adj, grad):
        """Path-replay adjoint of cast_rays(current_sample_in_block, pass_idx=pass_idx).

        adj: [B,H,W] float64 CUDA tensor (dLoss / d film cell); grad: [P] float64
        CUDA tensor, P = sum(param_count()), into which the gradient is ADDED."""
        import torch
        self.flush()
        c = self.config
        if adj.dtype != torch.float64 or tuple(adj.shape) != (c.bands, c.height, c.width) or not adj.is_contiguous():
            raise ValueError("adj must be a contiguous float64 [B, H, W] tensor")
        if grad.dtype != torch.float64 or grad.numel() != sum(self.param_count()) or not grad.is_contiguous():
            raise ValueError("grad must be a contiguous float64 tensor of param_count() entries")
        self._check(self.lib.ts_adjoint_pass(self._ctx, int(pass_idx) & 0xFFFFFFFF, int(current_sample_in_block),
                                             ctypes.c_void_p(adj.data_ptr()), ctypes.c_void_p(grad.data_ptr()),
                                             _stream()))

    def adjoint_passes(self, first_band, num_passes, first_pass, adj, grad):
        """adjoint_pass over num_passes consecutive passes in one launch."""
        import torch
        self.flush()
        c = self.config
        if adj.dtype != torch.float64 or tuple(adj.shape) != (c.bands, c.height, c.width) or not adj.is_contiguous():
            raise ValueError("adj must be a contiguous float64 [B, H, W] tensor")
        if grad.dtype != torch.float64 or grad.numel() != sum(self.param_count()) or not grad.is_contiguous():
            raise ValueError("grad must be a contiguous float64 tensor of param_count() entries")
        self._check(self.lib.ts_adjoint_passes(self._ctx, int(first_pass) & 0xFFFFFFFF, int(num_passes),
                                               int(first_band), ctypes.c_void_p(adj.data_ptr()),
                                               ctypes.c_void_p(grad.data_ptr()), _stream()))

    def check_device(self):
        """Raise if a kernel reported an error bit since the last check (synchronises)."""
        self.flush()
        bits = ctypes.c_uint32()
        self._check(self.lib.ts_check_device(self._ctx, ctypes.byref(bits)))
        return bits.value
