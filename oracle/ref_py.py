"""ctypes front end of the reference harness (oracle/ref_harness/ref_harness.cu).

TEST INFRASTRUCTURE: the reference's own KKT, Schur, dz kernels and qdldl
helper, compiled from the reference's sources, used as a parity oracle for
the CUDA product and for the C restatement in oracle.c.  The library is built
by `make -C oracle ref` when the reference tree is present; it is one library
per compiled-in velocity cost (QD_COST 1e-4: the reference's logged runs;
1e-2: the synthetic tracking problems).  Device arguments are torch CUDA
tensors (float32 / int32, contiguous).
"""
import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
_LIBS = {}


def lib_path(qd_cost: float) -> str:
    tag = {1e-4: "1e-4", 1e-2: "1e-2"}[qd_cost]
    return os.path.join(HERE, "_ref", f"libgptref_qd{tag}.so")


def available(qd_cost: float = 1e-4) -> bool:
    return os.path.exists(lib_path(qd_cost))


def load(qd_cost: float = 1e-4):
    if qd_cost in _LIBS:
        return _LIBS[qd_cost]
    L = C.CDLL(lib_path(qd_cost))
    vp, u32, f32, i32 = C.c_void_p, C.c_uint32, C.c_float, C.c_int
    sig = {
        "refh_form_kkt": [u32, f32, i32, vp, vp, vp, vp, vp, vp, vp],
        "refh_form_schur": [u32, f32, vp, vp, vp, vp, vp, vp, vp],
        "refh_form_schur_qdl": [u32, f32, vp, vp, vp, vp, vp, vp],
        "refh_prep_csr": [u32, vp, vp],
        "refh_compute_dz": [u32, vp, vp, vp, vp, vp],
        "refh_qdldl_solve": [u32, vp, vp, vp, vp, vp],
    }
    for name, args in sig.items():
        f = getattr(L, name)
        f.argtypes = args
        f.restype = i32
    _LIBS[qd_cost] = L
    return L


def _p(t):
    return None if t is None else C.c_void_p(t.data_ptr())


def _check(rc, what):
    if rc != 0:
        raise RuntimeError(f"reference harness {what}: error {rc}")


class Reference:
    """The reference's kernels for one compiled-in cost setting."""

    def __init__(self, qd_cost: float = 1e-4):
        self.L = load(qd_cost)

    def form_kkt(self, N, dt, integrator, G, Cm, g, c, eePos, xs, xu):
        _check(self.L.refh_form_kkt(N, dt, integrator, _p(G), _p(Cm), _p(g), _p(c), _p(eePos), _p(xs), _p(xu)),
               "form_kkt")

    def form_schur(self, N, rho, G, Cm, g, c, S, Pinv, gamma):
        """S, Pinv, gamma in the reference's 3-block layout; G is overwritten with Ginv."""
        _check(self.L.refh_form_schur(N, rho, _p(G), _p(Cm), _p(g), _p(c), _p(S), _p(Pinv), _p(gamma)),
               "form_schur")

    def form_schur_qdl(self, N, rho, G, Cm, g, c, val, gamma):
        _check(self.L.refh_form_schur_qdl(N, rho, _p(G), _p(Cm), _p(g), _p(c), _p(val), _p(gamma)),
               "form_schur_qdl")

    def prep_csr(self, N, col_ptr, row_ind):
        _check(self.L.refh_prep_csr(N, _p(col_ptr), _p(row_ind)), "prep_csr")

    def compute_dz(self, N, Ginv, Cm, g, lam, dz):
        _check(self.L.refh_compute_dz(N, _p(Ginv), _p(Cm), _p(g), _p(lam), _p(dz)), "compute_dz")

    def qdldl_solve(self, N, col_ptr, row_ind, val, gamma, lam):
        """Host numpy arrays (int32, int32, float32, float32, float32 out)."""
        f = lambda a: a.ctypes.data_as(C.c_void_p)
        _check(self.L.refh_qdldl_solve(N, f(col_ptr), f(row_ind), f(val), f(gamma), f(lam)), "qdldl_solve")
