"""ctypes view of libgli_b200's C ABI (include/gli_b200.h).

The struct layouts are those of the reference headers (include/range.h,
grid.h, gausslet.h, nuclear_integrals.h, kinetic_integrals.h,
eri_integrals.h, erida_integrals.h), which libgli_b200 keeps unchanged.
Loading fails loudly when the shared library has not been built.
"""
import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
# GLI_B200_LIBRARY selects another build of the library (the debug build
# libgli_b200_debug.so with its device bounds checks); default the release build
LIB_PATH = os.environ.get("GLI_B200_LIBRARY") or os.path.join(HERE, "libgli_b200.so")

glong = C.c_int64
dptr = C.POINTER(C.c_double)
lptr = C.POINTER(glong)

GLI_FORM_FP64 = 0
GLI_FORM_MIXED = 1
GLI_KIND_ERIDA = 0
GLI_KIND_ERI = 1


class Range(C.Structure):
    _fields_ = [("istart", glong), ("num", glong)]


class Grid(C.Structure):
    _fields_ = [("coord_range", Range * 3)]


class Point(C.Structure):
    _fields_ = [("c", glong * 3)]


class GaussletData(C.Structure):
    _fields_ = [("coefficients", dptr), ("indices", Range)]


class Nucleus(C.Structure):
    _fields_ = [("pos", C.c_double * 3), ("charge", C.c_int)]


class Kinetic(C.Structure):
    _fields_ = [("integral_values", dptr), ("grid", Grid)]


class Nuclear(C.Structure):
    _fields_ = [("integral_values", dptr), ("grid", Grid), ("nuclei", C.POINTER(Nucleus)), ("num_nuclei", C.c_int)]


class SparseIndices(C.Structure):
    """struct sparse_eri_indices / sparse_erida_indices (same layout)."""
    _fields_ = [("indices", lptr), ("num", glong), ("grid", Grid)]


class SparseIntegrals(C.Structure):
    """struct sparse_eri_gausslet_integrals / sparse_erida_gausslet_integrals."""
    _fields_ = [("integral_values", dptr), ("indices", lptr), ("num_entries", glong), ("grid", Grid)]


EXPORTS = [
    # reference API (include/{kinetic,nuclear,eri,erida}_integrals.h, symmetry.h)
    "compute_kinetic_gausslet_integral", "compute_kinetic_gausslet_integrals", "delete_kinetic_gausslet_integrals",
    "compute_nuclear_gausslet_integral", "compute_nuclear_gausslet_integrals", "delete_nuclear_gausslet_integrals",
    "compute_eri_gausslet_integral", "minimum_octahedral_orbit_eri_tensor_index",
    "enumerate_symmetry_reduced_eri_indices", "delete_sparse_eri_indices", "compute_sparse_eri_gausslet_integrals",
    "sparse_eri_gausslet_integrals_get_value", "project_sparse_eri_gausslet_integrals", "fill_dense_eri_tensor",
    "apply_sparse_eri_tensor", "delete_sparse_eri_gausslet_integrals",
    "compute_erida_gausslet_integral", "minimum_octahedral_orbit_erida_tensor_index",
    "enumerate_symmetry_reduced_erida_indices", "delete_sparse_erida_indices",
    "compute_sparse_erida_gausslet_integrals", "sparse_erida_gausslet_integrals_get_value",
    "project_sparse_erida_gausslet_integrals", "fill_dense_erida_matrix", "delete_sparse_erida_gausslet_integrals",
    "evaluate_octahedral_grid_permutations",
    # extensions
    "gli_b200_last_error", "gli_b200_last_error_message", "gli_b200_device_count", "gli_b200_set_device",
    "gli_b200_version", "gli_b200_sparse_values_dev", "gli_b200_sparse_values_dev_async",
    "gli_b200_sparse_values_wait", "gli_b200_sparse_values", "gli_b200_enumerate_dev",
    "gli_b200_free_dev", "gli_b200_set_timing", "gli_b200_last_stage_times", "gli_b200_last_stage_c_times",
    "gli_b200_last_plan",
    "gli_b200_last_paths", "gli_b200_last_screening", "gli_b200_clear_caches", "gli_b200_measure_fp64_peak",
    "gli_b200_kinetic_matrix_noalloc", "gli_b200_launch_count", "gli_b200_dgemm_sliced_dev",
    "gli_b200_nuclear_batch_dev", "gli_b200_nuclear_batch", "gli_b200_last_nuclear_batch", "gli_b200_autotune_report",
    "gli_b200_autotune_selftest", "gli_b200_surrogate_train", "gli_b200_surrogate_free", "gli_b200_surrogate_info",
    "gli_b200_surrogate_params", "gli_b200_erida_surrogate_values", "gli_b200_mlp_loss_grad",
    "gli_b200_mlp_param_count",
    # HDF5 subset (include/hdf5.h, include/hdf5_util.h)
    "gli_b200_h5_fopen", "gli_b200_h5_fcreate", "gli_b200_h5_fclose", "get_hdf5_dataset_ndims",
    "get_hdf5_dataset_dims", "read_hdf5_dataset", "write_hdf5_dataset", "get_hdf5_attribute_dims",
    "read_hdf5_attribute", "write_hdf5_scalar_attribute", "write_hdf5_vector_attribute",
]

# element type ids of include/hdf5.h
H5T_NATIVE_DOUBLE = 0x7f000001
H5T_NATIVE_LLONG = 0x7f000002
H5T_NATIVE_INT = 0x7f000003
H5T_IEEE_F64LE = 0x7f000011
H5T_STD_I64LE = 0x7f000012
H5T_STD_I32LE = 0x7f000013


def load(path=LIB_PATH):
    if not os.path.exists(path):
        raise ImportError(f"libgli_b200.so not built ({path}); run python -m gausslectronitegrate_b200.build")
    L = C.CDLL(path)
    P = C.POINTER
    L.compute_kinetic_gausslet_integral.argtypes = [P(GaussletData), P(Point)]
    L.compute_kinetic_gausslet_integral.restype = C.c_double
    L.compute_kinetic_gausslet_integrals.argtypes = [P(GaussletData), P(Grid), P(Kinetic)]
    L.delete_kinetic_gausslet_integrals.argtypes = [P(Kinetic)]
    L.compute_nuclear_gausslet_integral.argtypes = [P(GaussletData), P(Point), P(Nucleus), C.c_int, C.c_double]
    L.compute_nuclear_gausslet_integral.restype = C.c_double
    L.compute_nuclear_gausslet_integrals.argtypes = [P(GaussletData), P(Grid), P(Nucleus), C.c_int, C.c_double,
                                                     P(Nuclear)]
    L.delete_nuclear_gausslet_integrals.argtypes = [P(Nuclear)]
    for kind in ("eri", "erida"):
        getattr(L, f"compute_{kind}_gausslet_integral").argtypes = [P(GaussletData), P(Point), C.c_double]
        getattr(L, f"compute_{kind}_gausslet_integral").restype = C.c_double
        getattr(L, f"enumerate_symmetry_reduced_{kind}_indices").argtypes = [P(Grid), P(SparseIndices)]
        getattr(L, f"delete_sparse_{kind}_indices").argtypes = [P(SparseIndices)]
        getattr(L, f"compute_sparse_{kind}_gausslet_integrals").argtypes = [
            P(GaussletData), P(Grid), lptr, glong, C.c_double, P(SparseIntegrals)]
        getattr(L, f"sparse_{kind}_gausslet_integrals_get_value").argtypes = [P(SparseIntegrals), glong]
        getattr(L, f"sparse_{kind}_gausslet_integrals_get_value").restype = C.c_double
        getattr(L, f"project_sparse_{kind}_gausslet_integrals").argtypes = [P(SparseIntegrals), dptr, glong, dptr]
        getattr(L, f"delete_sparse_{kind}_gausslet_integrals").argtypes = [P(SparseIntegrals)]
    L.minimum_octahedral_orbit_eri_tensor_index.argtypes = [glong, P(lptr), glong, glong, glong, glong]
    L.minimum_octahedral_orbit_eri_tensor_index.restype = glong
    L.minimum_octahedral_orbit_erida_tensor_index.argtypes = [glong, P(lptr), glong, glong]
    L.minimum_octahedral_orbit_erida_tensor_index.restype = glong
    L.fill_dense_eri_tensor.argtypes = [P(SparseIntegrals), P(Grid), dptr]
    L.fill_dense_erida_matrix.argtypes = [P(SparseIntegrals), P(Grid), dptr]
    L.apply_sparse_eri_tensor.argtypes = [P(SparseIntegrals), dptr, glong, dptr]
    L.evaluate_octahedral_grid_permutations.argtypes = [P(Grid), P(lptr)]
    L.gli_b200_last_error.restype = C.c_int
    L.gli_b200_last_error_message.restype = C.c_char_p
    L.gli_b200_device_count.restype = C.c_int
    L.gli_b200_set_device.argtypes = [C.c_int]
    L.gli_b200_version.restype = C.c_char_p
    L.gli_b200_sparse_values_dev.argtypes = [C.c_int, dptr, glong, P(Grid), C.c_void_p, glong, C.c_double, C.c_int,
                                             C.c_void_p, C.c_void_p]
    L.gli_b200_sparse_values_dev_async.argtypes = [C.c_int, dptr, glong, P(Grid), C.c_void_p, glong, C.c_double,
                                                   C.c_int, C.c_void_p, C.c_void_p, P(glong)]
    L.gli_b200_sparse_values_wait.argtypes = [glong]
    L.gli_b200_sparse_values.argtypes = [C.c_int, P(GaussletData), P(Grid), lptr, glong, C.c_double, C.c_int, dptr]
    L.gli_b200_enumerate_dev.argtypes = [C.c_int, P(Grid), P(C.c_void_p), P(glong), C.c_void_p]
    L.gli_b200_free_dev.argtypes = [C.c_void_p, C.c_void_p]
    L.gli_b200_set_timing.argtypes = [C.c_int]
    L.gli_b200_last_stage_times.argtypes = [P(C.c_float), P(glong)]
    L.gli_b200_last_stage_c_times.argtypes = [P(C.c_float)]
    L.gli_b200_last_plan.argtypes = [P(glong)]
    L.gli_b200_last_paths.argtypes = [P(C.c_int)]
    L.gli_b200_last_screening.argtypes = [P(C.c_double)]
    hid = C.c_int64
    L.gli_b200_h5_fopen.argtypes = [C.c_char_p, C.c_uint, hid]
    L.gli_b200_h5_fopen.restype = hid
    L.gli_b200_h5_fcreate.argtypes = [C.c_char_p, C.c_uint, hid, hid]
    L.gli_b200_h5_fcreate.restype = hid
    L.gli_b200_h5_fclose.argtypes = [hid]
    L.get_hdf5_dataset_ndims.argtypes = [hid, C.c_char_p, C.c_void_p]
    for fn in ("get_hdf5_dataset_dims", "get_hdf5_attribute_dims"):
        getattr(L, fn).argtypes = [hid, C.c_char_p, C.c_void_p]
    for fn in ("read_hdf5_dataset", "read_hdf5_attribute"):
        getattr(L, fn).argtypes = [hid, C.c_char_p, hid, C.c_void_p]
    L.write_hdf5_dataset.argtypes = [hid, C.c_char_p, C.c_int, C.c_void_p, hid, hid, C.c_void_p]
    L.write_hdf5_scalar_attribute.argtypes = [hid, C.c_char_p, hid, hid, C.c_void_p]
    L.write_hdf5_vector_attribute.argtypes = [hid, C.c_char_p, hid, hid, glong, C.c_void_p]
    L.gli_b200_measure_fp64_peak.argtypes = [P(C.c_double)]
    L.gli_b200_kinetic_matrix_noalloc.argtypes = [C.c_void_p, glong, P(Grid), C.c_void_p, C.c_void_p]
    L.gli_b200_kinetic_matrix_noalloc.restype = C.c_int
    L.gli_b200_launch_count.restype = C.c_longlong
    L.gli_b200_dgemm_sliced_dev.argtypes = [C.c_void_p, glong, C.c_void_p, glong, C.c_void_p, glong, glong, glong, glong,
                                            C.c_void_p]
    L.gli_b200_dgemm_sliced_dev.restype = C.c_int
    L.gli_b200_nuclear_batch_dev.argtypes = [P(GaussletData), glong, P(Grid), lptr, P(Nucleus), C.c_double, C.c_int,
                                             P(C.c_void_p), C.c_void_p]
    L.gli_b200_nuclear_batch_dev.restype = C.c_int
    L.gli_b200_nuclear_batch.argtypes = [P(GaussletData), glong, P(Grid), lptr, P(Nucleus), C.c_double, C.c_int,
                                         P(C.c_void_p)]
    L.gli_b200_nuclear_batch.restype = C.c_int
    L.gli_b200_last_nuclear_batch.argtypes = [P(glong)]
    L.gli_b200_last_nuclear_batch.restype = None
    L.gli_b200_autotune_report.argtypes = [C.c_char_p, glong]
    L.gli_b200_autotune_report.restype = glong
    L.gli_b200_autotune_selftest.restype = C.c_int
    L.gli_b200_surrogate_train.argtypes = [P(GaussletData), C.c_double, C.c_double, C.c_int, C.c_double, C.c_double,
                                           C.c_ulonglong, P(C.c_void_p)]
    L.gli_b200_surrogate_train.restype = C.c_int
    L.gli_b200_surrogate_free.argtypes = [C.c_void_p]
    L.gli_b200_surrogate_free.restype = None
    L.gli_b200_surrogate_info.argtypes = [C.c_void_p, P(C.c_double)]
    L.gli_b200_surrogate_info.restype = C.c_int
    L.gli_b200_surrogate_params.argtypes = [C.c_void_p, P(C.c_float), glong]
    L.gli_b200_surrogate_params.restype = glong
    L.gli_b200_erida_surrogate_values.argtypes = [C.c_void_p, P(GaussletData), P(Grid), lptr, glong, C.c_double,
                                                  C.c_double, C.c_ulonglong, C.c_double, dptr, dptr, glong]
    L.gli_b200_erida_surrogate_values.restype = C.c_int
    L.gli_b200_mlp_loss_grad.argtypes = [P(C.c_float), P(C.c_float), P(C.c_float), P(C.c_float), glong,
                                         P(C.c_float), P(C.c_float)]
    L.gli_b200_mlp_loss_grad.restype = C.c_int
    L.gli_b200_mlp_param_count.restype = C.c_int
    return L
