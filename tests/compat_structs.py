"""ctypes mirrors of BaryTree's driver structs (the reference's
src/particles/struct_particles.h:5-27 and src/run_params/struct_run_params.h:7-31),
shared by the compatibility tests."""
import ctypes

_dp = ctypes.POINTER(ctypes.c_double)
_ip = ctypes.POINTER(ctypes.c_int)


class Particles(ctypes.Structure):
    _fields_ = [("num", ctypes.c_int), ("x", _dp), ("y", _dp), ("z", _dp), ("q", _dp), ("w", _dp),
                ("ibeg", _ip), ("iend", _ip), ("order", _ip),
                ("sources_w_dummy", ctypes.c_int), ("targets_q_dummy", ctypes.c_int),
                ("targets_x_duplicate", ctypes.c_int), ("targets_y_duplicate", ctypes.c_int),
                ("targets_z_duplicate", ctypes.c_int), ("targets_q_duplicate", ctypes.c_int)]


class RunParams(ctypes.Structure):
    _fields_ = [("kernel", ctypes.c_int), ("num_kernel_params", ctypes.c_int), ("kernel_params", _dp),
                ("approximation", ctypes.c_int), ("singularity", ctypes.c_int), ("compute_type", ctypes.c_int),
                ("theta", ctypes.c_double), ("size_check_factor", ctypes.c_double),
                ("interp_degree", ctypes.c_int), ("interp_pts_per_cluster", ctypes.c_int),
                ("interp_charges_per_cluster", ctypes.c_int), ("interp_weights_per_cluster", ctypes.c_int),
                ("max_per_source_leaf", ctypes.c_int), ("max_per_target_leaf", ctypes.c_int),
                ("beta", ctypes.c_double), ("verbosity", ctypes.c_int)]


def declare(lib):
    """argtypes of the driver functions on a library that exports them."""
    rp = ctypes.POINTER(RunParams)
    pp = ctypes.POINTER(Particles)
    lib.RunParams_Setup.argtypes = (ctypes.POINTER(rp), ctypes.c_int, ctypes.c_int, _dp, ctypes.c_int, ctypes.c_int,
                                    ctypes.c_int, ctypes.c_double, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                    ctypes.c_double, ctypes.c_double, ctypes.c_int)
    lib.RunParams_Setup.restype = None
    lib.RunParams_Free.argtypes = (ctypes.POINTER(rp),)
    lib.RunParams_Free.restype = None
    lib.RunParams_Validate.argtypes = (rp,)
    lib.RunParams_Validate.restype = None
    for fn in (lib.treedriver, lib.directdriver):
        fn.argtypes = (pp, pp, rp, _dp, _dp)
        fn.restype = None
    return lib


def particles(x, y, z, q, w=None):
    """A Particles struct over numpy arrays (kept alive by the caller)."""
    p = Particles()
    p.num = len(x)
    p.x, p.y, p.z, p.q = (a.ctypes.data_as(_dp) for a in (x, y, z, q))
    p.w = w.ctypes.data_as(_dp) if w is not None else None
    return p


def fields(rp):
    """The struct's fields as a dict (kernel parameters as a tuple)."""
    d = {name: getattr(rp, name) for name, _ in RunParams._fields_ if name != "kernel_params"}
    d["kernel_params"] = tuple(rp.kernel_params[i] for i in range(rp.num_kernel_params))
    return d
