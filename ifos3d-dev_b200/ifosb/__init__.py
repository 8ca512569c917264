"""Python host binding of the B200 IFOS3D wavefield engine.

Thin ctypes layer over the C ABI in ``include/ifos_b200.h`` (library
``ifos3d-dev_b200/lib/libifos_b200.so``). There is no CPU fallback: if the CUDA
library is missing or no GPU is present, the calls raise.

The names and argument meanings mirror the reference's driver
(src/ifos3d.c): a forward batch, residual(), the back-propagation, gradient_F.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

PKG_DIR = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB_PATH = os.path.join(PKG_DIR, "lib", "libifos_b200.so")

OK, EARG, ECUDA, ENOMEM, EUNSTABLE, ESTATE, ENODEV, ETOOBIG, EIO = 0, 1, 2, 3, 4, 5, 6, 7, 8
_NAMES = {EARG: "EARG", ECUDA: "ECUDA", ENOMEM: "ENOMEM", EUNSTABLE: "EUNSTABLE", ESTATE: "ESTATE", ENODEV: "ENODEV",
          ETOOBIG: "ETOOBIG", EIO: "EIO"}
NOALLOC_MAX_TRACES = 65536

F_VX, F_VY, F_VZ, F_SXX, F_SYY, F_SZZ, F_SXY, F_SYZ, F_SXZ = range(9)
F_DFT_FWD, F_DFT_BACK = 100, 200


class IfosbError(RuntimeError):
    def __init__(self, code, msg=""):
        super().__init__(f"ifosb error {_NAMES.get(code, code)}: {msg}")
        self.code = code


class Params(C.Structure):
    _fields_ = [
        ("nx", C.c_int), ("ny", C.c_int), ("nz", C.c_int),
        ("dx", C.c_float), ("dy", C.c_float), ("dz", C.c_float),
        ("dt", C.c_float), ("nt", C.c_int), ("time", C.c_float),
        ("fdorder", C.c_int), ("fdcoeff", C.c_int), ("free_surf", C.c_int), ("abs_type", C.c_int),
        ("fw", C.c_int), ("nmech", C.c_int), ("ndt", C.c_int), ("ndtshift", C.c_int),
        ("alpha", C.c_float), ("beta", C.c_float),
    ]


class Shot(C.Structure):
    _fields_ = [("nsrc", C.c_int), ("srcpos", C.c_void_p), ("signals", C.c_void_p)]


def build_library(force: bool = False) -> str:
    """Compile the CUDA library in-tree (nvcc, sm_100a). Returns the .so path."""
    if force or not os.path.exists(LIB_PATH):
        subprocess.run(["make", "-s", "-C", PKG_DIR], check=True)
    return LIB_PATH


_lib = None


def lib():
    """Load libifos_b200.so (raises if it is missing — no fallback path exists)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise FileNotFoundError(f"{LIB_PATH} is missing: build it with `make -C {PKG_DIR}`")
        L = C.CDLL(LIB_PATH)
        vp = C.c_void_p
        sig = {
            "ifosb_create": (C.c_int, [C.POINTER(Params), C.c_int, C.c_int, C.POINTER(vp)]),
            "ifosb_destroy": (None, [vp]),
            "ifosb_last_error": (C.c_char_p, [vp]),
            "ifosb_device_bytes": (C.c_longlong, [vp]),
            "ifosb_set_cpml": (C.c_int, [vp, vp]),
            "ifosb_set_model": (C.c_int, [vp, vp, vp, vp, vp, vp, vp]),
            "ifosb_set_receivers": (C.c_int, [vp, C.c_int, vp]),
            "ifosb_set_frequencies": (C.c_int, [vp, C.c_int, vp, C.c_int]),
            "ifosb_forward": (C.c_int, [vp, C.c_int, C.POINTER(Shot), vp]),
            "ifosb_residual": (C.c_int, [vp, vp, vp, vp]),
            "ifosb_adjoint": (C.c_int, [vp, vp]),
            "ifosb_gradient": (C.c_int, [vp]),
            "ifosb_gradient_td": (C.c_int, [vp, C.c_int, vp]),
            "ifosb_get_gradient_q": (C.c_int, [vp, vp]),
            "ifosb_zero_gradient": (C.c_int, [vp]),
            "ifosb_get_gradient": (C.c_int, [vp, vp, vp]),
            "ifosb_shot_gradient": (C.c_int, [vp, C.c_int, C.POINTER(Shot), vp, vp]),
            "ifosb_get_field": (C.c_int, [vp, C.c_int, C.c_int, vp]),
            "ifosb_set_launch_mode": (C.c_int, [vp, C.c_int]),
            "ifosb_last_launch_count": (C.c_longlong, [vp]),
            "ifosb_graph_captures": (C.c_longlong, [vp]),
            "ifosb_cpml_coeff": (C.c_int, [C.POINTER(Params), C.c_float, C.c_float, vp]),
            "ifosb_wavelet": (C.c_int, [C.POINTER(Params), C.c_int, C.c_int, vp, vp]),
            "ifosb_nsamples": (C.c_int, [C.POINTER(Params)]),
            "ifosb_moduli": (C.c_int, [C.POINTER(Params), C.c_longlong, vp, vp, vp, C.c_float, vp, vp, vp, vp, vp, vp]),
            "ifosb_set_profiling": (C.c_int, [vp, C.c_int]),
            "ifosb_kernel_times": (C.c_int, [vp, C.POINTER(C.c_double), C.POINTER(C.c_double), C.POINTER(C.c_int)]),
            "ifosb_set_stream": (C.c_int, [vp, vp]),
            "ifosb_autotune": (C.c_int, [vp, C.c_int, C.POINTER(Shot), C.c_int, vp]),
            "ifosb_set_launch_shape": (C.c_int, [vp, C.c_int, vp]),
            "ifosb_residual_noalloc": (C.c_int, [C.c_int, C.c_int, C.c_int, C.c_float, vp, vp, vp, vp, vp]),
            "ifosb_optim_create": (C.c_int, [C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.POINTER(vp)]),
            "ifosb_optim_destroy": (None, [vp]),
            "ifosb_optim_last_error": (C.c_char_p, [vp]),
            "ifosb_conjugate": (C.c_int, [vp, vp, C.c_int, vp]),
            "ifosb_lbfgs_savegrad": (C.c_int, [vp, vp]),
            "ifosb_lbfgs": (C.c_int, [vp, vp, C.c_int]),
            "ifosb_modelupdate": (C.c_int, [vp, vp, vp, vp, vp, C.c_float, vp, C.c_float, C.c_float, C.c_float,
                                            C.c_int, C.c_int]),
            "ifosb_lbfgs_history": (C.c_int, [vp, vp, vp, vp]),
            "ifosb_steplength": (C.c_int, [vp, vp, C.c_int, C.c_int, C.c_double, vp]),
            "ifosb_constant_boundary": (C.c_int, [vp, vp, vp, vp, C.c_int]),
            "ifosb_precon_grad": (C.c_int, [vp, vp, C.c_int, C.c_int, C.c_int, C.c_float, C.c_float, C.c_float,
                                            C.c_int, vp, C.c_int, vp]),
            "ifosb_write_seis": (C.c_int, [C.c_char_p, C.c_int, vp, C.c_int, C.c_int, vp, vp, vp, C.c_float,
                                           C.c_float, C.c_float, C.c_int, C.c_float, C.c_int, C.c_int]),
            "ifosb_merge_seis": (C.c_int, [C.c_char_p, C.c_int, C.POINTER(C.c_char_p), C.c_int,
                                           C.POINTER(C.c_int)]),
            "ifosb_read_seis": (C.c_int, [C.c_char_p, vp, C.c_int, C.c_int]),
            "ifosb_read_seis_split": (C.c_int, [C.c_char_p, vp, C.c_int, vp, C.c_int]),
            "ifosb_write_model": (C.c_int, [C.c_char_p, C.c_int, C.c_int, C.c_int, C.c_int, vp, vp, vp, C.c_int,
                                            C.c_int, C.c_int, C.c_int]),
            "ifosb_write_gradient": (C.c_int, [C.c_char_p, C.c_float, C.c_int, C.c_int, C.c_int, C.c_int, vp,
                                               C.c_int, C.c_int, C.c_int, C.c_int]),
            "ifosb_filt_seis": (C.c_int, [vp, C.c_int, C.c_int, C.c_float, C.c_float, C.c_int, C.c_int]),
            "ifosb_hessian_green": (C.c_int, [vp, C.c_int, vp, vp]),
            "ifosb_hessian": (C.c_int, [vp]),
            "ifosb_zero_hessian": (C.c_int, [vp]),
            "ifosb_get_hessian": (C.c_int, [vp, vp]),
            "ifosb_read_hessian": (C.c_int, [C.c_char_p, C.c_float, C.c_int, C.c_int, C.c_int, C.c_int, C.c_float,
                                             C.c_float, C.c_float, vp]),
            "ifosb_hess_apply": (C.c_int, [vp, vp, vp, vp, C.c_int, C.c_float, C.c_float, C.c_float]),
            "ifosb_resample": (C.c_int, [vp, C.c_int, C.c_int, C.c_int, C.c_float, C.c_float, C.c_float, vp,
                                         C.c_int, C.c_int, C.c_int, C.c_float, C.c_float, C.c_float]),
            "ifosb_set_seismo": (C.c_int, [vp, C.c_int]),
            "ifosb_set_wait_test": (C.c_int, [vp, C.c_longlong, C.c_int, C.c_int]),
            "ifosb_set_surface_moduli": (C.c_int, [vp, vp, vp]),
            "ifosb_vjp_exact": (C.c_int, [vp, C.c_int, vp, vp]),
            "ifosb_vjp_exact_moduli": (C.c_int, [vp, C.c_int, vp, vp]),
            "ifosb_set_td_checkpoints": (C.c_int, [vp, C.c_int]),
        }
        for name, (res, args) in sig.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def exported_symbols():
    """Names of the C-ABI entry points this binding expects."""
    return [
        "ifosb_create", "ifosb_destroy", "ifosb_last_error", "ifosb_device_bytes", "ifosb_set_cpml",
        "ifosb_set_model", "ifosb_set_receivers", "ifosb_set_frequencies", "ifosb_forward", "ifosb_residual",
        "ifosb_adjoint", "ifosb_gradient", "ifosb_zero_gradient", "ifosb_get_gradient", "ifosb_shot_gradient",
        "ifosb_get_field", "ifosb_set_launch_mode", "ifosb_last_launch_count", "ifosb_graph_captures", "ifosb_cpml_coeff",
        "ifosb_wavelet", "ifosb_nsamples", "ifosb_moduli", "ifosb_set_profiling", "ifosb_kernel_times",
        "ifosb_set_stream", "ifosb_autotune", "ifosb_set_launch_shape", "ifosb_residual_noalloc", "ifosb_optim_create", "ifosb_optim_destroy",
        "ifosb_optim_last_error", "ifosb_conjugate", "ifosb_lbfgs_savegrad", "ifosb_lbfgs", "ifosb_modelupdate",
        "ifosb_lbfgs_history", "ifosb_steplength", "ifosb_precon_grad", "ifosb_constant_boundary",
        "ifosb_write_seis", "ifosb_merge_seis", "ifosb_read_seis", "ifosb_read_seis_split",
        "ifosb_write_model", "ifosb_write_gradient", "ifosb_filt_seis", "ifosb_hessian_green", "ifosb_hessian",
        "ifosb_zero_hessian", "ifosb_get_hessian", "ifosb_read_hessian", "ifosb_hess_apply", "ifosb_resample",
        "ifosb_set_seismo", "ifosb_gradient_td", "ifosb_get_gradient_q", "ifosb_set_wait_test",
        "ifosb_set_surface_moduli", "ifosb_vjp_exact", "ifosb_vjp_exact_moduli", "ifosb_set_td_checkpoints",
    ]


def _p(a):
    return None if a is None else a.ctypes.data


def _f32(a):
    return None if a is None else np.ascontiguousarray(a, dtype=np.float32)


def _is_tensor(a) -> bool:
    return hasattr(a, "data_ptr") and hasattr(a, "is_cuda")


def _traces(a):
    """(keep-alive object, address) of observed traces: a numpy array (host) or a
    contiguous float32 CUDA tensor (device-resident traces, no host copy)."""
    if _is_tensor(a):
        import torch
        if not (a.is_cuda and a.dtype == torch.float32 and a.is_contiguous()):
            raise ValueError("device traces must be a contiguous float32 CUDA tensor")
        return a, a.data_ptr()
    h = _f32(a)
    return h, _p(h)


def make_params(nx, ny, nz, dh=1.0, dt=1e-4, nt=100, fdcoeff=2, free_surf=1, fw=10, nmech=0, ndt=1, ndtshift=0,
                alpha=0.0, beta=0.0, dx=None, dy=None, dz=None) -> Params:
    """Parameters as the reference derives them: TIME=(NT-1)*DT in float (ifos3d.c:176-177)."""
    dtf = np.float32(dt)
    return Params(nx=nx, ny=ny, nz=nz, dx=dx or dh, dy=dy or dh, dz=dz or dh, dt=dtf, nt=nt,
                  time=np.float32(np.float32(nt - 1) * dtf), fdorder=4, fdcoeff=fdcoeff, free_surf=free_surf,
                  abs_type=1, fw=fw, nmech=nmech, ndt=ndt, ndtshift=ndtshift, alpha=alpha, beta=beta)


def nsamples(p: Params) -> int:
    return lib().ifosb_nsamples(C.byref(p))


def residual_noalloc(nshots: int, ntr: int, ns: int, dt: float, d_syn: int, d_obs: int, d_diff: int,
                     d_misfit: int, stream: int = 0) -> int:
    """ifosb_residual_noalloc on device addresses (ints); enqueued on `stream`
    (a cudaStream_t as int), not waited for. Returns the status code."""
    return lib().ifosb_residual_noalloc(nshots, ntr, ns, dt, C.c_void_p(d_syn), C.c_void_p(d_obs),
                                        C.c_void_p(d_diff), C.c_void_p(d_misfit), C.c_void_p(stream or None))


def cpml_coeff(p: Params, vppml: float, fpml: float) -> np.ndarray:
    out = np.zeros((18, 2 * p.fw), np.float32)
    _check(None, lib().ifosb_cpml_coeff(C.byref(p), vppml, fpml, _p(out)))
    return out


def wavelet(p: Params, shape: int, srcpos) -> np.ndarray:
    srcpos = _f32(np.atleast_2d(srcpos))
    out = np.zeros((srcpos.shape[0], p.nt), np.float32)
    _check(None, lib().ifosb_wavelet(C.byref(p), shape, srcpos.shape[0], _p(srcpos), _p(out)))
    return out


def moduli(p: Params, vp, vs, rho, tau=0.0, fl=None):
    """readmod() arithmetic: returns dict(rho, pi, u, taus, taup, eta) (interior arrays)."""
    vp, vs, rho = _f32(vp), _f32(vs), _f32(rho)
    n = vp.size
    pi, u = np.zeros_like(vp), np.zeros_like(vp)
    L = p.nmech
    taus = np.zeros_like(vp) if L else None
    taup = np.zeros_like(vp) if L else None
    eta = np.zeros(max(L, 1), np.float32)
    fla = _f32(fl) if L else None
    _check(None, lib().ifosb_moduli(C.byref(p), n, _p(vp), _p(vs), _p(rho), tau, _p(fla), _p(pi), _p(u),
                                    _p(taus), _p(taup), _p(eta)))
    return dict(rho=rho, pi=pi, u=u, taus=taus, taup=taup, eta=eta[:L] if L else None)


def ghost_wrap(a) -> np.ndarray:
    """The model with one ghost layer as matcopy() leaves it on one rank: a
    periodic wrap (src/matcopy.c:31-327, receives from MPI_PROC_NULL are no-ops)."""
    return np.ascontiguousarray(np.pad(np.asarray(a, np.float32), 1, mode="wrap"))


def _check(eng, rc):
    if rc != OK:
        msg = lib().ifosb_last_error(eng).decode() if eng else ""
        raise IfosbError(rc, msg)


class Engine:
    """One device-resident problem (model, CPML, receivers, frequencies) and a
    batch of up to ``max_shots`` shots."""

    def __init__(self, p: Params, max_shots: int = 1, max_nf: int = 0):
        self.p = p
        self.max_shots = max_shots
        h = C.c_void_p()
        rc = lib().ifosb_create(C.byref(p), max_shots, max_nf, C.byref(h))
        if rc != OK:
            raise IfosbError(rc, "ifosb_create")
        self.h = h
        self.ntr = 0
        self.ns = nsamples(p)
        self.nf = 0

    def close(self):
        if getattr(self, "h", None):
            lib().ifosb_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _c(self, rc):
        _check(self.h, rc)

    @property
    def device_bytes(self) -> int:
        return lib().ifosb_device_bytes(self.h)

    def set_cpml(self, coeff):
        coeff = _f32(coeff)
        self._c(lib().ifosb_set_cpml(self.h, _p(coeff)))

    def set_model(self, rho, pi, u, taus=None, taup=None, eta=None, ghosted=False):
        """Interior [NY][NX][NZ] arrays (wrapped here like matcopy on one rank) or,
        with ghosted=True, the caller's own [NY+2][NX+2][NZ+2] arrays."""
        w = (lambda a: _f32(a)) if ghosted else (lambda a: None if a is None else ghost_wrap(a))
        arrs = [w(rho), w(pi), w(u), w(taus), w(taup), _f32(eta)]
        self._keep = arrs
        self._c(lib().ifosb_set_model(self.h, *[_p(a) for a in arrs]))

    def set_surface_moduli(self, pi=None, u=None, ghosted=False):
        """Moduli of the elastic free surface at j = 1 when they differ from the
        propagation model's (the reference's step-length forwards); None restores
        the model's own."""
        if pi is None:
            self._c(lib().ifosb_set_surface_moduli(self.h, None, None))
            return
        w = (lambda a: _f32(a)) if ghosted else ghost_wrap
        arrs = [w(pi), w(u)]
        self._c(lib().ifosb_set_surface_moduli(self.h, _p(arrs[0]), _p(arrs[1])))

    def set_receivers(self, recpos):
        rec = np.ascontiguousarray(recpos, dtype=np.int32).reshape(-1, 3)
        self._c(lib().ifosb_set_receivers(self.h, rec.shape[0], _p(rec)))
        self.ntr = rec.shape[0]

    def set_frequencies(self, finv, ntast=1):
        f = _f32(finv) if finv is not None and len(finv) else None
        nf = 0 if f is None else len(f)
        self._c(lib().ifosb_set_frequencies(self.h, nf, _p(f), ntast))
        self.nf = nf

    def set_wait_test(self, wait_ns: int = 1_000_000_000, kernel: int = 0, stop_plane: int = -1):
        """Failure-path test knobs (ifosb_set_wait_test): the TMA kernels' mbarrier
        wait limit, and the kernel (1 velocity, 2 stress) whose producer warp stops
        issuing loads at chunk iteration stop_plane. Defaults restore normal runs."""
        self._c(lib().ifosb_set_wait_test(self.h, int(wait_ns), kernel, stop_plane))

    def set_launch_mode(self, mode: int):
        self._c(lib().ifosb_set_launch_mode(self.h, mode))

    @property
    def graph_captures(self) -> int:
        return lib().ifosb_graph_captures(self.h)

    @property
    def launch_count(self) -> int:
        return lib().ifosb_last_launch_count(self.h)

    def set_profiling(self, on: bool):
        self._c(lib().ifosb_set_profiling(self.h, 1 if on else 0))

    def kernel_times(self):
        """(velocity ms, stress ms, steps) of the last profiled time loop."""
        v, s, n = C.c_double(), C.c_double(), C.c_int()
        self._c(lib().ifosb_kernel_times(self.h, C.byref(v), C.byref(s), C.byref(n)))
        return v.value, s.value, n.value

    def set_stream(self, stream_handle):
        """Launch on the caller's cudaStream_t (an int handle, e.g. torch's stream.cuda_stream)."""
        self._c(lib().ifosb_set_stream(self.h, C.c_void_p(stream_handle) if stream_handle else None))

    @staticmethod
    def _shots(shots):
        keep, arr = [], (Shot * len(shots))()
        for s, (srcpos, signals) in enumerate(shots):
            sp = _f32(np.atleast_2d(srcpos))
            sg = _f32(np.atleast_2d(signals))
            keep += [sp, sg]
            arr[s] = Shot(sp.shape[0], _p(sp), _p(sg))
        return arr, keep

    SEISMO_COMPONENTS = {1: ("vx", "vy", "vz"), 2: ("p",), 3: ("div", "curl"), 4: ("vx", "vy", "vz", "p", "div", "curl")}

    def set_seismo(self, seismo):
        """SEISMO 1-4: which components forward() records (SEISMO_COMPONENTS)."""
        self._c(lib().ifosb_set_seismo(self.h, seismo))
        self.seismo = seismo

    def forward(self, shots, want_sections=True):
        """shots: list of (srcpos[nsrc][7], signals[nsrc][NT]). Returns
        [nshots][ncomp][ntr][ns] (ncomp = 3 for SEISMO 1) or None."""
        arr, keep = self._shots(shots)
        ncomp = len(self.SEISMO_COMPONENTS[getattr(self, "seismo", 1)])
        out = np.zeros((len(shots), ncomp, self.ntr, self.ns), np.float32) if (want_sections and self.ntr) else None
        self._c(lib().ifosb_forward(self.h, len(shots), arr, _p(out)))
        return out

    def autotune(self, shots, steps=20):
        """Pick the launch shapes for batches of len(shots) shots; returns a dict with
        the y planes per CTA chunk and L2 prefetch distance of each kernel."""
        arr, keep = self._shots(shots)
        shape = np.zeros(4, np.int32)
        self._c(lib().ifosb_autotune(self.h, len(shots), arr, steps, _p(shape)))
        return {"velocity": {"y_planes_per_cta": int(shape[0]), "l2_prefetch_planes": int(shape[1])},
                "stress": {"y_planes_per_cta": int(shape[2]), "l2_prefetch_planes": int(shape[3])}}

    def set_launch_shape(self, nshots, shape):
        """shape: the dict autotune() returns, or [cy_vel, l2_vel, cy_str, l2_str]."""
        if isinstance(shape, dict):
            shape = [shape["velocity"]["y_planes_per_cta"], shape["velocity"]["l2_prefetch_planes"],
                     shape["stress"]["y_planes_per_cta"], shape["stress"]["l2_prefetch_planes"]]
        arr = np.ascontiguousarray(shape, np.int32)
        self._c(lib().ifosb_set_launch_shape(self.h, nshots, _p(arr)))

    def residual(self, obs, want_l2_ref=False):
        """obs: host traces (numpy) or device-resident ones (a float32 CUDA tensor)."""
        obs, addr = _traces(obs)
        nsh = obs.shape[0]
        mis = np.zeros(nsh, np.float64)
        l2 = np.zeros(nsh, np.float32) if want_l2_ref else None
        self._c(lib().ifosb_residual(self.h, addr, _p(mis), _p(l2)))
        return (mis, l2) if want_l2_ref else mis

    def adjoint(self, diff=None):
        d = _f32(diff)
        self._c(lib().ifosb_adjoint(self.h, _p(d)))

    def gradient(self):
        self._c(lib().ifosb_gradient(self.h))

    def zero_gradient(self):
        self._c(lib().ifosb_zero_gradient(self.h))

    def get_gradient_q(self):
        """Viscoelastic: FP64 gradients with respect to taup and taus, [2, NY, NX, NZ]
        (gradient_F's sign: minus the misfit gradient)."""
        g = np.zeros((2, self.p.ny, self.p.nx, self.p.nz), np.float64)
        self._c(lib().ifosb_get_gradient_q(self.h, _p(g)))
        return g

    def gradient_td(self, interval):
        """Time-domain kernels of the last forward batch and its residual with a
        checkpoint every `interval` steps: float64 [4, NY, NX, NZ] = rho, lambda,
        mu and the zero-frequency product (sums over the batch's shots)."""
        k = np.zeros((4, self.p.ny, self.p.nx, self.p.nz), np.float64)
        self._c(lib().ifosb_gradient_td(self.h, int(interval), _p(k)))
        return k

    def set_td_checkpoints(self, interval):
        """interval > 0: following forwards also keep the time-domain checkpoints of
        that interval, so that gradient_td(interval) skips its re-run of the
        forward; 0: off."""
        self._c(lib().ifosb_set_td_checkpoints(self.h, int(interval)))

    def vjp_exact(self, interval=25, want_grad=True, moduli=False):
        """The exact discrete gradient of the misfit of the last forward batch and its
        residual: (the gradient summed over the batch's shots, or None without
        want_grad; the FP64 misfit per shot). The time loop runs in FP64 with a
        checkpoint every `interval` steps; explosive sources. moduli=False (elastic
        engines): d misfit / d (vp, vs, rho), float64 [3, NY, NX, NZ]. moduli=True
        (any L): d misfit / d (rho, pi, u, taus, taup) of the model set_model received,
        float64 [5, NY, NX, NZ]."""
        nq = 5 if moduli else 3
        g = np.zeros((nq, self.p.ny, self.p.nx, self.p.nz), np.float64) if want_grad else None
        mis = np.zeros(max(1, self.max_shots), np.float64)
        fn = lib().ifosb_vjp_exact_moduli if moduli else lib().ifosb_vjp_exact
        self._c(fn(self.h, int(interval), _p(g), _p(mis)))
        return g, mis

    # -- approximate Hessian (hess_F) -----------------------------------------
    def hessian_green(self, rec_ids, signals):
        """Green's functions of receivers rec_ids: a y-force signals[q] ([NT]; one
        row shared by all when 1-D) at receiver rec_ids[q]."""
        r = np.ascontiguousarray(rec_ids, np.int32)
        sig = np.asarray(signals, np.float32)
        if sig.ndim == 1:
            sig = np.broadcast_to(sig, (len(r), sig.size))
        sig = np.ascontiguousarray(sig)
        if sig.shape != (len(r), self.p.nt):
            raise IfosbError(EARG, f"signals of shape {sig.shape}, expected ({len(r)}, NT={self.p.nt})")
        self._c(lib().ifosb_hessian_green(self.h, len(r), _p(r), _p(sig)))

    def hessian(self):
        """Add the last forward batch's hess_F contributions to the device Hessian."""
        self._c(lib().ifosb_hessian(self.h))

    def zero_hessian(self):
        self._c(lib().ifosb_zero_hessian(self.h))

    def get_hessian(self):
        h = np.zeros((3, self.p.ny, self.p.nx, self.p.nz), np.float32)
        self._c(lib().ifosb_get_hessian(self.h, _p(h)))
        return h

    def get_gradient(self, fp64=False, out=None):
        """The accumulated gradient [3, NY, NX, NZ]: a new host array, or copied into
        `out` (a host array, or a contiguous CUDA tensor of the right dtype)."""
        shape = (3, self.p.ny, self.p.nx, self.p.nz)
        if out is None:
            out = np.zeros(shape, np.float64 if fp64 else np.float32)
        if _is_tensor(out):
            import torch
            want = torch.float64 if fp64 else torch.float32
            if not (out.is_cuda and out.dtype == want and out.is_contiguous() and tuple(out.shape) == shape):
                raise ValueError(f"gradient tensor must be a contiguous CUDA {want} tensor of shape {shape}")
            addr = out.data_ptr()
        else:
            if out.dtype != (np.float64 if fp64 else np.float32) or not out.flags.c_contiguous or out.shape != shape:
                raise ValueError("gradient array of the wrong dtype, layout or shape")
            addr = _p(out)
        if fp64:
            self._c(lib().ifosb_get_gradient(self.h, None, addr))
        else:
            self._c(lib().ifosb_get_gradient(self.h, addr, None))
        return out

    def shot_gradient(self, shots, obs):
        """forward + residual + adjoint + gradient of a batch; obs host (numpy) or
        device-resident (float32 CUDA tensor). Returns the FP64 misfit per shot."""
        arr, keep = self._shots(shots)
        obs, addr = _traces(obs)
        mis = np.zeros(len(shots), np.float64)
        self._c(lib().ifosb_shot_gradient(self.h, len(shots), arr, addr, _p(mis)))
        return mis

    def get_field(self, shot: int, field: int) -> np.ndarray:
        out = np.zeros((self.p.ny + 5, self.p.nx + 4, self.p.nz + 4), np.float32)
        self._c(lib().ifosb_get_field(self.h, shot, field, _p(out)))
        return out

    def get_state(self, shot: int = 0) -> np.ndarray:
        return np.stack([self.get_field(shot, f) for f in range(9)])

    def get_dft(self, shot: int = 0, back: bool = False) -> np.ndarray:
        base = F_DFT_BACK if back else F_DFT_FWD
        return np.stack([np.stack([self.get_field(shot, base + c * self.nf + l) for l in range(self.nf)])
                         for c in range(6)])


class Optimizer:
    """The reference's model-space update state on the device (CG priors,
    L-BFGS history) with FP64 dot products: conjugate(), lbfgs_savegrad(),
    lbfgs(), modelupdate() of src/conjugategrad.c, src/lbfgs_save.c,
    src/lbfgs.c, src/modelupdate.c. Gradients are [3][NY][NX][NZ] float32
    (updated in place); models the ghosted [NY+2][NX+2][NZ+2] float32 arrays."""

    def __init__(self, nx: int, ny: int, nz: int, numpar: int = 1, bfgsnum: int = 0):
        self.shape = (ny, nx, nz)
        self.numpar, self.bfgsnum = numpar, bfgsnum
        h = C.c_void_p()
        rc = lib().ifosb_optim_create(nx, ny, nz, numpar, bfgsnum, C.byref(h))
        if rc != OK:
            raise IfosbError(rc, "ifosb_optim_create")
        self.h = h

    def close(self):
        if getattr(self, "h", None):
            lib().ifosb_optim_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _c(self, rc):
        if rc != OK:
            raise IfosbError(rc, lib().ifosb_optim_last_error(self.h).decode())

    def _grad(self, grad):
        if not (isinstance(grad, np.ndarray) and grad.dtype == np.float32 and grad.flags.c_contiguous
                and grad.shape == (3,) + self.shape):
            raise ValueError(f"gradient must be a C-contiguous float32 array of shape {(3,) + self.shape}")
        return grad

    def conjugate(self, grad, cdf: int) -> np.ndarray:
        beta = np.zeros(3, np.float64)
        self._c(lib().ifosb_conjugate(self.h, _p(self._grad(grad)), cdf, _p(beta)))
        return beta

    def lbfgs_savegrad(self, grad):
        self._c(lib().ifosb_lbfgs_savegrad(self.h, _p(self._grad(grad))))

    def lbfgs(self, grad, it_group: int):
        self._c(lib().ifosb_lbfgs(self.h, _p(self._grad(grad)), it_group))

    def modelupdate(self, grad, rho, pi, u, step, weight, vp0, vs0, rho0, lbfgs=False, it_group=1):
        mshape = tuple(s + 2 for s in self.shape)
        for a in (rho, pi, u):
            if not (isinstance(a, np.ndarray) and a.dtype == np.float32 and a.flags.c_contiguous and a.shape == mshape):
                raise ValueError(f"model arrays must be C-contiguous float32 of shape {mshape}")
        w = np.ascontiguousarray(weight, np.float32)
        self._c(lib().ifosb_modelupdate(self.h, _p(self._grad(grad)), _p(rho), _p(pi), _p(u), step, _p(w), vp0, vs0,
                                        rho0, int(bool(lbfgs)), it_group))

    def precon_grad(self, grad, damptype, free_surf, fw, dh, srcpos_m, recpos):
        """precon_grad on grad [3][NY][NX][NZ] in place; srcpos_m [nsrc][3] metres,
        recpos [ntr][3] grid indices; dh = (DX, DY, DZ)."""
        src = np.ascontiguousarray(np.atleast_2d(srcpos_m), np.float32) if len(srcpos_m) else None
        rec = np.ascontiguousarray(np.atleast_2d(recpos), np.int32) if len(recpos) else None
        self._c(lib().ifosb_precon_grad(self.h, _p(self._grad(grad)), damptype, int(bool(free_surf)), fw, dh[0], dh[1],
                                        dh[2], 0 if src is None else src.shape[0], _p(src),
                                        0 if rec is None else rec.shape[0], _p(rec)))

    def hess_apply(self, grad, hess, water, lbfgs=False, vp0=0.0, vs0=0.0, rho0=0.0):
        """hess_apply: grad [3][NY][NX][NZ] in place divided by hess + water[c]
        (scaled first by VP0, VS0, RHO0 with L-BFGS)."""
        h = self._grad(np.ascontiguousarray(hess, np.float32))
        w = np.ascontiguousarray(water, np.float32)
        self._c(lib().ifosb_hess_apply(self.h, _p(self._grad(grad)), _p(h), _p(w), int(bool(lbfgs)), vp0, vs0, rho0))

    def constant_boundary(self, rho, pi, u, fw):
        """constant_boundary on the ghosted model arrays in place."""
        mshape = tuple(s + 2 for s in self.shape)
        for a in (rho, pi, u):
            if not (isinstance(a, np.ndarray) and a.dtype == np.float32 and a.flags.c_contiguous and a.shape == mshape):
                raise ValueError(f"model arrays must be C-contiguous float32 of shape {mshape}")
        self._c(lib().ifosb_constant_boundary(self.h, _p(rho), _p(pi), _p(u), fw))

    def history(self):
        nn = self.numpar * int(np.prod(self.shape))
        s = np.zeros((self.bfgsnum, nn), np.float64)
        y = np.zeros((self.bfgsnum, nn), np.float64)
        sc = np.zeros(self.bfgsnum, np.float64)
        self._c(lib().ifosb_lbfgs_history(self.h, _p(s), _p(y), _p(sc)))
        return s, y, sc


def steplength(L2, step, lbfgs=False, it_group=1, teststep=0.0):
    """steplength() in FP64. L2[4], step[5] float64 arrays updated in place;
    returns the parabola coefficients (a, b, c)."""
    if not (isinstance(L2, np.ndarray) and L2.dtype == np.float64 and L2.size >= 4):
        raise ValueError("L2 must be a float64 array of 4")
    if not (isinstance(step, np.ndarray) and step.dtype == np.float64 and step.size >= 5):
        raise ValueError("step must be a float64 array of 5")
    abc = np.zeros(3, np.float64)
    _check(None, lib().ifosb_steplength(_p(L2), _p(step), int(bool(lbfgs)), it_group, teststep, _p(abc)))
    return abc


def q_gradient(gradq, taup, taus, q):
    """d/dQ from get_gradient_q's taup / taus gradients when both tau scale as 1/Q
    (the tau method): -(taup d/dtaup + taus d/dtaus) / Q, per cell (q scalar or
    [NY, NX, NZ])."""
    g = np.asarray(gradq, np.float64)
    return -(np.asarray(taup, np.float64) * g[0] + np.asarray(taus, np.float64) * g[1]) / np.asarray(q, np.float64)
