"""ctypes bindings of the native libraries.

``host()`` — libdtfe_host.so (tessellator, planning; CPU only).
``gpu()``  — libdtfe_gpu.so (CUDA kernels + C ABI of include/dtfe_gpu.h).

There is no fallback: if a library is missing or fails to load, the call
raises.  The product path never substitutes a CPU implementation for a
kernel.
"""
from __future__ import annotations

import ctypes as C
import os

from . import build as _build

_host = None
_gpu = None

c_i32p = C.POINTER(C.c_int32)
c_i64p = C.POINTER(C.c_int64)


class Subbox(C.Structure):
    """dtfe_subbox (include/dtfe_gpu.h)."""
    _fields_ = [
        ("vert_offset", C.c_int64), ("n_verts", C.c_int64),
        ("tet_offset", C.c_int64), ("n_tets", C.c_int64),
        ("tile_origin", C.c_int32 * 3), ("tile_dims", C.c_int32 * 3),
        ("coord_offset", C.c_int64 * 3),
        ("dx", C.c_float * 3), ("lo", C.c_float * 3),
        ("part_no", C.c_int32), ("reserved", C.c_int32),
    ]


class DepositBox(C.Structure):
    """dtfe_deposit_box."""
    _fields_ = [("particle_offset", C.c_int64), ("n_particles", C.c_int64), ("region", C.c_float * 6),
                ("tile_origin", C.c_int32 * 3), ("tile_dims", C.c_int32 * 3)]


class PlanView(C.Structure):
    """dtfe_plan_view (include/dtfe_host.h)."""
    _fields_ = [("kind", C.c_int32), ("grid", C.c_int32 * 3), ("rho_bar", C.c_double), ("padding", C.c_float * 6),
                ("n_verts", C.c_int64), ("n_tets", C.c_int64), ("n_boxes", C.c_int32), ("n_scalars", C.c_int32),
                ("tet_v", C.c_void_p), ("tet_n", C.c_void_p), ("xyz", C.c_void_p), ("src", C.c_void_p),
                ("weight", C.c_void_p), ("velocity", C.c_void_p), ("scalar", C.c_void_p),
                ("boxes", C.c_void_p), ("regions", C.c_void_p), ("xs", C.c_void_p), ("ys", C.c_void_p),
                ("zs", C.c_void_p),
                ("n_xs", C.c_int64), ("n_ys", C.c_int64), ("n_zs", C.c_int64),
                ("n_particles", C.c_int64), ("dep_pos", C.c_void_p), ("dep_weight", C.c_void_p),
                ("dep_velocity", C.c_void_p), ("dep_src", C.c_void_p), ("n_dep_boxes", C.c_int32),
                ("dep_boxes", C.c_void_p), ("region", C.c_float * 6)]


class PlanOptions(C.Structure):
    """dtfe_plan_options (include/dtfe_host.h)."""
    _fields_ = [("n_parts", C.c_int32), ("padding_mode", C.c_int32), ("padding_particles", C.c_float),
                ("padding", C.c_float * 6), ("region_on", C.c_int32), ("region", C.c_float * 6),
                ("partition_on", C.c_int32), ("partition", C.c_int32 * 3), ("part_no", C.c_int32),
                ("average_density", C.c_double)]


PAD_PARTICLES, PAD_RELATIVE, PAD_ABSOLUTE = 0, 1, 2


class InterpOpts(C.Structure):
    """dtfe_interp_opts."""
    _fields_ = [("method", C.c_int32), ("n_samples", C.c_int32), ("seed", C.c_uint64),
                ("fields", C.c_uint32), ("flags", C.c_uint32)]


class Status(C.Structure):
    """dtfe_status."""
    _fields_ = [("n_samples_located", C.c_int64), ("n_outside", C.c_int64),
                ("n_walk_failures", C.c_int64), ("n_walk_steps", C.c_int64),
                ("n_exact_tests", C.c_int64), ("n_ties", C.c_int64)]

    def as_dict(self) -> dict:
        return {k: int(getattr(self, k)) for k, _ in self._fields_}


class Config(C.Structure):
    """dtfe_config."""
    _fields_ = [("device", C.c_int32), ("n_scalars", C.c_int32),
                ("max_walk_steps", C.c_int32), ("reserved", C.c_int32)]


# status codes (include/dtfe_gpu.h)
OK, ERR_ARG, ERR_CUDA, ERR_ALLOC, ERR_STATE, ERR_WALK, ERR_DEGENERATE, ERR_NO_DEVICE, ERR_TOO_LARGE, ERR_IO = range(10)
NUM_FIELDS = 9
NOALLOC_MAX_VERTS = 1 << 20
FIELD_SLOTS = {
    "density": 0, "velocity": 1, "velocity_gradient": 2, "velocity_divergence": 3,
    "velocity_shear": 4, "velocity_vorticity": 5, "velocity_std": 6,
    "scalar": 7, "scalar_gradient": 8,
}
METHOD_CENTRE, METHOD_TETRAHEDRA, METHOD_MONTE_CARLO, METHOD_EQUIDISTANT = 0, 1, 2, 3
FLAG_FIX_VALUE_INTERP = 1
FLAG_FIX_OUTSIDE_RASTER = 2


def field_components(slot: int, n_scalars: int) -> int:
    return [1, 3, 9, 1, 5, 3, 1, n_scalars, 3 * n_scalars][slot]


class DTFEError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"DTFE error {code}: {msg}")
        self.code = code


def _load(path: str) -> C.CDLL:
    if not os.path.exists(path):
        raise OSError(f"native library missing: {path} (run __graft_entry__.build())")
    return C.CDLL(path)


def host() -> C.CDLL:
    global _host
    if _host is None:
        lib = _load(os.path.join(_build.BUILD, "libdtfe_host.so"))
        vp = C.c_void_p
        lib.dtfe_tessellate.argtypes = [vp, C.c_int64, C.c_uint64, C.c_int, C.POINTER(vp)]
        lib.dtfe_tessellate.restype = C.c_int
        lib.dtfe_tessellate_batch.argtypes = [C.c_int, C.POINTER(vp), c_i64p, C.c_uint64, C.c_int,
                                              C.POINTER(vp), C.POINTER(C.c_int)]
        lib.dtfe_tessellate_batch.restype = None
        lib.dtfe_tess_sizes.argtypes = [vp, c_i64p, c_i64p, c_i64p]
        lib.dtfe_tess_export.argtypes = [vp, vp, vp, vp]
        lib.dtfe_tess_release.argtypes = [vp]
        for name in ("dtfe_orient", "dtfe_orient_exact"):
            getattr(lib, name).argtypes = [vp] * 4
            getattr(lib, name).restype = C.c_int
        for name in ("dtfe_insphere", "dtfe_insphere_exact"):
            getattr(lib, name).argtypes = [vp] * 5
            getattr(lib, name).restype = C.c_int
        lib.dtfe_padding_length.argtypes = [C.c_int, C.c_float, C.c_int64, vp, vp, vp]
        lib.dtfe_padding_length.restype = None
        lib.dtfe_average_density.argtypes = [vp, C.c_int64]
        lib.dtfe_average_density.restype = C.c_float
        lib.dtfe_select_in_box.argtypes = [vp, C.c_int64, vp, vp, C.c_int, vp, vp]
        lib.dtfe_select_in_box.restype = C.c_int64
        lib.dtfe_parallel_grid.argtypes = [C.c_int64, vp, vp]
        lib.dtfe_write_binary.argtypes = [C.c_char_p, vp, C.c_int64]
        lib.dtfe_write_binary.restype = C.c_int
        lib.dtfe_field_suffix.argtypes = [C.c_int32, C.c_int32]
        lib.dtfe_field_suffix.restype = C.c_char_p
        lib.dtfe_optimal_partition.argtypes = [vp, C.c_int64, vp, vp, vp, vp, vp]
        lib.dtfe_optimal_partition.restype = C.c_int
        lib.dtfe_axis_coords.argtypes = [C.c_float, C.c_float, C.c_int64, vp]
        lib.dtfe_tets_pack.argtypes = [vp, vp, C.c_int64, vp]
        lib.dtfe_tets_pack.restype = C.c_int64
        lib.dtfe_tets_unpack.argtypes = [vp, C.c_int64, vp, vp]
        lib.dtfe_tets_pack_vertices.argtypes = [vp, C.c_int64, vp]
        lib.dtfe_tets_pack_vertices.restype = C.c_int64
        lib.dtfe_tets_unpack_vertices.argtypes = [vp, C.c_int64, vp]
        lib.dtfe_plan_build.argtypes = [C.c_int, vp, vp, vp, vp, C.c_int32, C.c_int64, vp, C.c_int, vp, C.c_int32,
                                        C.c_float, C.c_double, C.POINTER(C.c_void_p)]
        lib.dtfe_plan_build_ex.argtypes = [C.c_int, vp, vp, vp, vp, C.c_int32, C.c_int64, vp, C.c_int, vp,
                                           C.POINTER(PlanOptions), C.POINTER(C.c_void_p)]
        lib.dtfe_plan_get.argtypes = [C.c_void_p, C.POINTER(PlanView)]
        lib.dtfe_plan_release.argtypes = [C.c_void_p]
        _host = lib
    return _host


def gpu() -> C.CDLL:
    global _gpu
    if _gpu is None:
        lib = _load(os.path.join(_build.BUILD, "libdtfe_gpu.so"))
        vp = C.c_void_p
        H = C.c_void_p
        lib.dtfe_last_error.restype = C.c_char_p
        lib.dtfe_gpu_create.argtypes = [C.POINTER(Config), C.POINTER(H)]
        lib.dtfe_gpu_destroy.argtypes = [H]
        lib.dtfe_gpu_upload.argtypes = [H, vp, vp, C.c_int64, vp, vp, vp, vp, C.c_int64]
        lib.dtfe_gpu_chain_uploads.argtypes = [H, H]
        lib.dtfe_gpu_upload_packed.argtypes = [H, vp, C.c_int64, vp, vp, vp, vp, C.c_int64]
        lib.dtfe_gpu_upload_packed_particles.argtypes = [H, vp, C.c_int64, vp, vp, vp, vp, C.c_int64, vp,
                                                         C.c_int64, vp]
        lib.dtfe_gpu_set_subboxes.argtypes = [H, C.c_int32, vp, vp, C.c_int64, vp, C.c_int64,
                                              vp, C.c_int64, vp]
        lib.dtfe_gpu_set_regions.argtypes = [H, C.c_int32, vp]
        lib.dtfe_gpu_vertex_density.argtypes = [H, C.c_double]
        lib.dtfe_gpu_interpolate.argtypes = [H, C.POINTER(InterpOpts), C.POINTER(vp), C.POINTER(Status)]
        lib.dtfe_gpu_interpolate_async.argtypes = [H, C.POINTER(InterpOpts), C.POINTER(vp)]
        lib.dtfe_gpu_interpolate_dev.argtypes = [H, C.POINTER(InterpOpts), C.POINTER(vp), C.POINTER(Status)]
        lib.dtfe_gpu_interpolate_dev_async.argtypes = [H, C.POINTER(InterpOpts), C.POINTER(vp)]
        lib.dtfe_gpu_interpolate_points.argtypes = [H, C.c_int64, vp, vp, C.POINTER(InterpOpts), C.POINTER(vp),
                                                    C.POINTER(C.c_int64)]
        lib.dtfe_gpu_interpolate_cone.argtypes = [H, vp, vp, vp, C.POINTER(InterpOpts), C.POINTER(vp)]
        lib.dtfe_gpu_average_points.argtypes = [H, C.c_int64, vp, vp, vp, C.POINTER(InterpOpts), C.POINTER(vp),
                                                C.POINTER(C.c_int64)]
        lib.dtfe_gpu_interpolate_cone_dev.argtypes = [H, vp, vp, vp, C.POINTER(InterpOpts), C.POINTER(vp)]
        lib.dtfe_gpu_write_binary_dev.argtypes = [H, C.c_char_p, vp, C.c_int64]
        lib.dtfe_gpu_select_in_box_dev.argtypes = [H, vp, C.c_int64, vp, vp, C.c_int, vp, vp, C.c_int64,
                                                   C.POINTER(C.c_int64)]
        lib.dtfe_gpu_download_vertex_density.argtypes = [H, vp]
        lib.dtfe_gpu_locate_points.argtypes = [H, C.c_int64, vp, C.c_int32, vp]
        lib.dtfe_gpu_download_located.argtypes = [H, vp]
        lib.dtfe_gpu_download_tets.argtypes = [H, vp, vp]
        lib.dtfe_gpu_tiles_gather_dev.argtypes = [H, C.c_int32, vp, vp, C.c_int32, vp, vp]
        lib.dtfe_gpu_tiles_scatter_dev.argtypes = [H, C.c_int32, vp, vp, C.c_int32, vp, vp]
        lib.dtfe_gpu_set_max_walk_steps.argtypes = [H, C.c_int32]
        lib.dtfe_gpu_stream.argtypes = [H]
        lib.dtfe_gpu_stream.restype = C.c_void_p
        lib.dtfe_gpu_synchronize.argtypes = [H]
        lib.dtfe_gpu_deposit.argtypes = [H, C.c_int32, vp, vp, vp, C.c_int64, C.c_int32, vp, vp, C.c_double, vp, vp]
        lib.dtfe_gpu_deposit_dev.argtypes = [H, C.c_int32, vp, vp, vp, C.c_int64, C.c_int32, vp, vp, C.c_double,
                                             vp, vp]
        lib.dtfe_gpu_deposit_resident.argtypes = [H, C.c_int32, vp, vp, vp, C.c_int64, C.c_int32, vp, vp,
                                                  C.c_double, vp, vp]
        lib.dtfe_gpu_graph_build.argtypes = [H, C.c_double, C.POINTER(InterpOpts), C.POINTER(vp)]
        lib.dtfe_gpu_graph_launch.argtypes = [H]
        lib.dtfe_gpu_read_status.argtypes = [H, C.POINTER(Status)]
        lib.dtfe_gpu_sph.argtypes = [H, C.c_int32, C.c_uint32, C.c_int32, C.c_double, vp, vp, vp]
        lib.dtfe_gpu_sph_dev.argtypes = [H, C.c_int32, C.c_uint32, C.c_int32, C.c_double, vp, vp, vp]
        lib.dtfe_gpu_adjoint_dev.argtypes = [H, vp, vp, vp, vp, vp, vp]
        lib.dtfe_gpu_deposit_adjoint_dev.argtypes = [H, vp, vp, vp]
        lib.dtfe_gpu_autotune.argtypes = [H, C.c_uint32, vp]
        lib.dtfe_gpu_set_variants.argtypes = [H, C.c_int32, C.c_int32]
        lib.dtfe_gpu_variant_counts.argtypes = [vp]
        lib.dtfe_vertex_density_noalloc.argtypes = [vp, vp, C.c_int64, vp, vp, C.c_int64, C.c_double, vp, vp]
        lib.dtfe_vertex_density_noalloc.restype = C.c_int
        lib.dtfe_gpu_tessellate.argtypes = [vp, C.c_int32, vp, vp, C.POINTER(vp)]
        lib.dtfe_gpu_tess_sizes.argtypes = [vp, vp, vp]
        lib.dtfe_gpu_tess_export.argtypes = [vp, vp, C.c_int32]
        lib.dtfe_gpu_tess_stats.argtypes = [vp, vp, C.c_int32]
        lib.dtfe_gpu_tess_release.argtypes = [vp]
        _gpu = lib
    return _gpu


def check(rc: int) -> None:
    if rc != OK:
        msg = gpu().dtfe_last_error().decode(errors="replace") if _gpu is not None else ""
        raise DTFEError(rc, msg)


def ptr(a) -> int:
    """Address of a numpy array or torch tensor (0 for None)."""
    if a is None:
        return 0
    if hasattr(a, "data_ptr"):
        return a.data_ptr()
    return a.ctypes.data
