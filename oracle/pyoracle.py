"""ctypes binding to the CPU oracle libraries — TEST INFRASTRUCTURE ONLY.

Loads either the reference build (``oracle/_ref/libifos_ref.so``: the reference's
own C functions driven by ``oracle/ref_harness.c``) or the C restatement
(``oracle/lib/libifos_oracle.so``). Both export the functions declared in
``oracle/ifos_oracle.h``. Imported only by tests/, ``__graft_entry__.smoke()`` and
the cpu_baseline leg of ``bench.py``; the CUDA product never touches it.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_LIB = os.path.join(HERE, "_ref", "libifos_ref.so")
ORC_LIB = os.path.join(HERE, "lib", "libifos_oracle.so")
# the reference checkout: IFOS_REFERENCE_SRC, else a sibling of this repository
REFERENCE_SRC = os.environ.get("IFOS_REFERENCE_SRC",
                               os.path.normpath(os.path.join(HERE, "..", "..", "reference")))


class IfoParams(C.Structure):
    _fields_ = [
        ("nx", C.c_int), ("ny", C.c_int), ("nz", C.c_int),
        ("dx", C.c_float), ("dy", C.c_float), ("dz", C.c_float),
        ("dt", C.c_float), ("nt", C.c_int), ("time", C.c_float),
        ("fdcoeff", C.c_int), ("free_surf", C.c_int), ("fw", C.c_int), ("nmech", C.c_int),
        ("ndt", C.c_int), ("ndtshift", C.c_int),
        ("vppml", C.c_float), ("fpml", C.c_float),
        ("alpha", C.c_float), ("beta", C.c_float),
        ("source_shape", C.c_int),
    ]


class IfoVelModel(C.Structure):
    _fields_ = [("vp", C.c_void_p), ("vs", C.c_void_p), ("rho", C.c_void_p),
                ("tau", C.c_float), ("fl", C.c_void_p)]


def build(which: str = "oracle") -> None:
    """Build ``oracle`` (the restatement, needs only gcc) or ``ref`` (needs the reference sources)."""
    subprocess.run(["make", "-s", "-C", HERE, which], check=True)


def have_ref() -> bool:
    return os.path.exists(REF_LIB)


def _ptr(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


def _f32(a):
    return None if a is None else np.ascontiguousarray(a, dtype=np.float32)


class Oracle:
    """One of the two CPU oracle implementations behind the same API."""

    def __init__(self, kind: str = "oracle", threads: int = 0):
        """kind "ref" (the reference build, single-threaded) or "oracle" (the
        restatement; its cell loops use `threads` OpenMP threads, 0 = all cores)."""
        path = REF_LIB if kind == "ref" else ORC_LIB
        if not os.path.exists(path):
            if kind == "ref" and not os.path.isdir(os.path.join(REFERENCE_SRC, "src")):
                raise FileNotFoundError(f"{path} missing and no reference sources to build it from")
            build("ref" if kind == "ref" else "oracle")
        self.kind = kind
        self.lib = C.CDLL(path)
        for name in ("ifo_readmod", "ifo_cpml_coeff", "ifo_wavelet", "ifo_av_mat", "ifo_forward",
                     "ifo_residual", "ifo_adjoint", "ifo_gradient", "ifo_nsamples"):
            getattr(self.lib, name).restype = C.c_int
        if hasattr(self.lib, "ifo_set_threads"):
            self.lib.ifo_set_threads.restype = None
            self.lib.ifo_set_threads.argtypes = [C.c_int]
            self.lib.ifo_set_threads(int(threads))

    # -- helpers ---------------------------------------------------------------
    @staticmethod
    def wshape(p: IfoParams):
        return (p.ny + 5, p.nx + 4, p.nz + 4)

    def nsamples(self, p: IfoParams) -> int:
        return self.lib.ifo_nsamples(C.byref(p))

    def readmod(self, p: IfoParams, vp, vs, rho, tau=0.0, fl=None):
        vp, vs, rho = _f32(vp), _f32(vs), _f32(rho)
        fl = _f32(fl if fl is not None else np.zeros(max(p.nmech, 1)))
        vm = IfoVelModel(_ptr(vp).value, _ptr(vs).value, _ptr(rho).value, tau, _ptr(fl).value)
        shp = vp.shape
        r, pi, u = (np.zeros(shp, np.float32) for _ in range(3))
        ts, tp = (np.zeros(shp, np.float32) for _ in range(2))
        eta = np.zeros(max(p.nmech, 1), np.float32)
        rc = self.lib.ifo_readmod(C.byref(p), C.byref(vm), _ptr(r), _ptr(pi), _ptr(u), _ptr(ts), _ptr(tp), _ptr(eta))
        assert rc == 0, rc
        return dict(rho=r, pi=pi, u=u, taus=ts if p.nmech else None, taup=tp if p.nmech else None,
                    eta=eta[:p.nmech] if p.nmech else None)

    def cpml_coeff(self, p: IfoParams):
        out = np.zeros((18, 2 * p.fw), np.float32)
        assert self.lib.ifo_cpml_coeff(C.byref(p), _ptr(out)) == 0
        return out

    def wavelet(self, p: IfoParams, srcpos):
        srcpos = _f32(srcpos)
        out = np.zeros((srcpos.shape[0], p.nt), np.float32)
        assert self.lib.ifo_wavelet(C.byref(p), srcpos.shape[0], _ptr(srcpos), _ptr(out)) == 0
        return out

    def av_mat(self, p: IfoParams, m):
        out = np.zeros((9, p.ny, p.nx, p.nz), np.float32)
        rc = self.lib.ifo_av_mat(C.byref(p), _ptr(_f32(m["rho"])), _ptr(_f32(m["pi"])), _ptr(_f32(m["u"])),
                                 _ptr(_f32(m.get("taus"))), _ptr(_f32(m.get("taup"))), _ptr(out))
        assert rc == 0
        return out

    def forward(self, p: IfoParams, m, cpml, srcpos, signals, recpos, finv=None, ntast=1,
                want_dft=False, want_state=False):
        ns = self.nsamples(p)
        recpos = np.ascontiguousarray(recpos, dtype=np.int32)
        srcpos, signals = _f32(srcpos), _f32(signals)
        nf = 0 if finv is None else len(finv)
        finv = _f32(finv) if nf else None
        sec = np.zeros((3, recpos.shape[0], ns), np.float32)
        dft = np.zeros((6, nf) + self.wshape(p), np.float32) if (want_dft and nf) else None
        st = np.zeros((9,) + self.wshape(p), np.float32) if want_state else None
        keep = [_f32(m["rho"]), _f32(m["pi"]), _f32(m["u"]), _f32(m.get("taus")), _f32(m.get("taup")),
                _f32(m.get("eta")), _f32(cpml)]
        rc = self.lib.ifo_forward(C.byref(p), *[_ptr(a) for a in keep], srcpos.shape[0], _ptr(srcpos), _ptr(signals),
                                  recpos.shape[0], _ptr(recpos), nf, _ptr(finv), ntast, _ptr(sec), _ptr(dft), _ptr(st))
        if rc:
            raise RuntimeError(f"ifo_forward rc={rc}")
        return dict(sections=sec, dft=dft, state=st)

    def forward_seismo(self, p: IfoParams, m, cpml, srcpos, signals, recpos, seismo):
        """The forward with SEISMO 1-4 (reference build): (v [3][ntr][ns], pdc [3][ntr][ns])."""
        ns = self.nsamples(p)
        recpos = np.ascontiguousarray(recpos, dtype=np.int32)
        srcpos, signals = _f32(srcpos), _f32(signals)
        sec = np.zeros((3, recpos.shape[0], ns), np.float32)
        pdc = np.zeros((3, recpos.shape[0], ns), np.float32)
        keep = [_f32(m["rho"]), _f32(m["pi"]), _f32(m["u"]), _f32(m.get("taus")), _f32(m.get("taup")),
                _f32(m.get("eta")), _f32(cpml)]
        rc = self.lib.ifo_forward_seismo(C.byref(p), *[_ptr(a) for a in keep], srcpos.shape[0], _ptr(srcpos),
                                         _ptr(signals), recpos.shape[0], _ptr(recpos), seismo, _ptr(sec), _ptr(pdc))
        if rc:
            raise RuntimeError(f"ifo_forward_seismo rc={rc}")
        return sec, pdc

    def residual(self, p: IfoParams, obs, syn):
        obs, syn = _f32(obs), _f32(syn)
        diff = np.zeros_like(syn)
        l2 = C.c_float(0.0)
        assert self.lib.ifo_residual(C.byref(p), syn.shape[1], _ptr(obs), _ptr(syn), _ptr(diff), C.byref(l2)) == 0
        return diff, float(l2.value)

    def adjoint(self, p: IfoParams, m, cpml, recpos, diff, finv, ntast=1, want_state=False):
        recpos = np.ascontiguousarray(recpos, dtype=np.int32)
        diff = _f32(diff)
        nf = len(finv)
        finv = _f32(finv)
        dft = np.zeros((6, nf) + self.wshape(p), np.float32)
        st = np.zeros((9,) + self.wshape(p), np.float32) if want_state else None
        keep = [_f32(m["rho"]), _f32(m["pi"]), _f32(m["u"]), _f32(m.get("taus")), _f32(m.get("taup")),
                _f32(m.get("eta")), _f32(cpml)]
        rc = self.lib.ifo_adjoint(C.byref(p), *[_ptr(a) for a in keep], recpos.shape[0], _ptr(recpos), _ptr(diff),
                                  nf, _ptr(finv), ntast, _ptr(dft), _ptr(st))
        if rc:
            raise RuntimeError(f"ifo_adjoint rc={rc}")
        return dict(dft=dft, state=st)

    def hessian(self, p: IfoParams, m, finv, dft_f, greens, hess=None):
        """hess_F of one shot (dft_f [6][nf][W]) against receivers' DFT fields
        greens [ngreen][6][nf][W], added to hess [3][ny][nx][nz] (reference build)."""
        h = np.zeros((3, p.ny, p.nx, p.nz), np.float32) if hess is None else np.ascontiguousarray(hess, np.float32).copy()
        finv = _f32(finv)
        greens = _f32(greens)
        rc = self.lib.ifo_hessian(C.byref(p), _ptr(_f32(m["rho"])), _ptr(_f32(m["pi"])), _ptr(_f32(m["u"])),
                                  len(finv), _ptr(finv), _ptr(_f32(dft_f)), greens.shape[0], _ptr(greens), _ptr(h))
        assert rc == 0
        return h

    def gradient(self, p: IfoParams, m, finv, dft_f, dft_b, grad=None):
        g = np.zeros((3, p.ny, p.nx, p.nz), np.float32) if grad is None else np.ascontiguousarray(grad, np.float32).copy()
        finv = _f32(finv)
        rc = self.lib.ifo_gradient(C.byref(p), _ptr(_f32(m["rho"])), _ptr(_f32(m["pi"])), _ptr(_f32(m["u"])),
                                   len(finv), _ptr(finv), _ptr(_f32(dft_f)), _ptr(_f32(dft_b)), _ptr(g))
        assert rc == 0
        return g
