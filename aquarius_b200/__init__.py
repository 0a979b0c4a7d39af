"""Python binding of the B200 CCSD engine (ctypes over libccsd_b200.so).

The C ABI (include/ccsd_b200.h) is the product boundary; this module mirrors it for
tests, benchmarks and Python callers:

    ctx = Context(device=0)
    ctx.set_spaces(nirrep=1, vrt=[v], occ=[o])
    H = ctx.hamiltonian_from_factor(B, eps)
    s = ctx.solver(H, conv_tol=1e-9, diis_order=8, precision="fp64")
    energy, conv, iters = s.run()

Every failing call raises CcsdError with the engine's message.  There is no
fallback: if the shared library or a CUDA device is missing, calls fail loudly.
"""
from __future__ import annotations

import ctypes
import itertools
import os
from pathlib import Path

import numpy as np

_HERE = Path(__file__).resolve().parent
# CCSD_B200_LIB points at another build of the library (e.g. a variant under test)
LIB_PATH = Path(os.environ["CCSD_B200_LIB"]) if os.environ.get("CCSD_B200_LIB") else _HERE / "libccsd_b200.so"

CCSD_OK = 0
STATUS = {
    0: "CCSD_OK", 1: "CCSD_ERR_ARG", 2: "CCSD_ERR_CUDA", 3: "CCSD_ERR_OOM", 4: "CCSD_ERR_PLAN",
    5: "CCSD_DIVERGED", 6: "CCSD_NOT_CONVERGED", 7: "CCSD_ERR_SINGULAR", 8: "CCSD_ERR_TIMEOUT",
    9: "CCSD_ERR_UNSUPPORTED",
}
PREC = {"fp64": 0, "split": 1, "split_i8": 2}   # split: BF16 slices; split_i8: INT8 slices
TENSOR_PACKED = 1
TENSOR_PLAIN = 2

# symbols declared in include/ccsd_b200.h
EXPORTS = [
    "ccsd_ctx_create", "ccsd_ctx_destroy", "ccsd_last_error", "ccsd_ctx_synchronize", "ccsd_ctx_device_bytes",
    "ccsd_ctx_launch_count", "ccsd_ctx_set_precision", "ccsd_ctx_set_profiling", "ccsd_ctx_profile_report",
    "ccsd_ctx_set_spaces", "ccsd_tensor_create",
    "ccsd_tensor_destroy", "ccsd_tensor_ndim", "ccsd_tensor_spin_cases", "ccsd_tensor_block_size",
    "ccsd_tensor_write_block", "ccsd_tensor_read_block", "ccsd_tensor_write", "ccsd_tensor_read", "ccsd_tensor_fill",
    "ccsd_contract", "ccsd_sum", "ccsd_scale", "ccsd_dot", "ccsd_norm", "ccsd_weight", "ccsd_options_default",
    "ccsd_hamiltonian_from_factor", "ccsd_hamiltonian_destroy", "ccsd_solver_create", "ccsd_solver_destroy",
    "ccsd_solver_mp2", "ccsd_solver_iterate", "ccsd_solver_iterate_async", "ccsd_solver_status", "ccsd_solver_run",
    "ccsd_solver_amplitudes", "ccsd_solver_flops", "ccsd_plan_query", "ccsd_synth_irreps", "ccsd_synth_problem",
    "ccsd_dot_batch_noalloc", "ccsd_hamiltonian_create", "ccsd_hamiltonian_from_integrals", "ccsd_fcidump_read",
    "ccsd_hamiltonian_from_fcidump", "ccsd_ctx_set_split_routing", "ccsd_ctx_split_launches",
    "ccsd_server_options_default", "ccsd_server_create", "ccsd_server_submit_synthetic", "ccsd_server_submit_factor",
    "ccsd_server_poll", "ccsd_server_wait", "ccsd_server_stats", "ccsd_server_destroy", "ccsd_solver_mode",
    "ccsd_rhf_hamiltonian_from_factor", "ccsd_rhf_hamiltonian_from_integrals", "ccsd_rhf_hamiltonian_destroy",
    "ccsd_rhf_solver_create", "ccsd_rhf_plan_query", "ccsd_hamiltonian_from_ao", "ccsd_rhf_hamiltonian_from_ao",
    "ccsd_rhf_solver_hbar", "ccsd_ctx_plan_flops", "ccsd_solver_hbar", "ccsd_lambda_solver_create",
    "ccsd_lambda_plan_query", "ccsd_ctx_plan_export", "ccsd_plan_export_solver",
    "ccsd_diis_create", "ccsd_diis_extrapolate", "ccsd_diis_coefficients", "ccsd_diis_destroy",
    "ccsd_slice_choice", "ccsd_solver_slice_report",
]


class CcsdError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"{STATUS.get(code, code)}: {msg}")
        self.code = code


class Options(ctypes.Structure):
    _fields_ = [
        ("conv_tol", ctypes.c_double), ("max_iter", ctypes.c_int), ("diis_order", ctypes.c_int),
        ("diis_start", ctypes.c_int), ("diis_damping", ctypes.c_double), ("precision", ctypes.c_int),
        ("slices", ctypes.c_int), ("use_graph", ctypes.c_int), ("refine_tol", ctypes.c_double),
        ("autotune_de", ctypes.c_double),
    ]


H_FIELDS = ["fAI", "fME", "fAE", "fMI", "VMNIJ", "VAMIJ", "VMNEJ", "VABIJ", "VMNEF", "VAMEI", "VAMEF", "VABEJ",
            "VABEF"]
# (nout, nin) per H block, {vrt, occ} order (src/operator/2eoperator.cxx:13-21)
H_SHAPES = {
    "fAI": ((1, 0), (0, 1)), "fME": ((0, 1), (1, 0)), "fAE": ((1, 0), (1, 0)), "fMI": ((0, 1), (0, 1)),
    "VMNIJ": ((0, 2), (0, 2)), "VAMIJ": ((1, 1), (0, 2)), "VMNEJ": ((0, 2), (1, 1)), "VABIJ": ((2, 0), (0, 2)),
    "VMNEF": ((0, 2), (2, 0)), "VAMEI": ((1, 1), (1, 1)), "VAMEF": ((1, 1), (2, 0)), "VABEJ": ((2, 0), (1, 1)),
    "VABEF": ((2, 0), (2, 0)),
}


class Hamiltonian(ctypes.Structure):
    _fields_ = [(f, ctypes.c_int32) for f in H_FIELDS]


# closed-shell spatial blocks (rhfccsd.cxx:19-30); VAIJB holds <ai|jb> at [a, i, b, j]
RHF_FIELDS = ["fAI", "fAB", "fIJ", "VABCD", "VABCI", "VABIJ", "VAIBJ", "VAIJB", "VAIJK", "VIJKL"]
RHF_SHAPES = {
    "fAI": ((1, 0), (0, 1)), "fAB": ((1, 0), (1, 0)), "fIJ": ((0, 1), (0, 1)), "VABCD": ((2, 0), (2, 0)),
    "VABCI": ((2, 0), (1, 1)), "VABIJ": ((2, 0), (0, 2)), "VAIBJ": ((1, 1), (1, 1)), "VAIJB": ((1, 1), (1, 1)),
    "VAIJK": ((1, 1), (0, 2)), "VIJKL": ((0, 2), (0, 2)),
}


class RHFHamiltonian(ctypes.Structure):
    _fields_ = [(f, ctypes.c_int32) for f in RHF_FIELDS]


# closed-shell Hbar intermediates (rhfccsd.cxx:110-186); W(Am,Ie) holds (a,m,i,e) at [a,m,e,i]
HBAR_SHAPES = {
    "FME": ((0, 1), (1, 0)), "FMI": ((0, 1), (0, 1)), "FAE": ((1, 0), (1, 0)), "WMNIJ": ((0, 2), (0, 2)),
    "WMNEJ": ((0, 2), (1, 1)), "WAMIJ": ((1, 1), (0, 2)), "WAMIE": ((1, 1), (1, 1)), "WAMEI": ((1, 1), (1, 1)),
    "WABEJ": ((2, 0), (1, 1)),
}


class RHFHbar(ctypes.Structure):
    _fields_ = [(f, ctypes.c_int32) for f in HBAR_SHAPES]


class ServerOptions(ctypes.Structure):
    _fields_ = [("device", ctypes.c_int), ("memory_budget", ctypes.c_int64), ("max_active", ctypes.c_int),
                ("pack_vvvv", ctypes.c_int), ("solve", Options)]


class ServerResult(ctypes.Structure):
    _fields_ = [("id", ctypes.c_int64), ("status", ctypes.c_int), ("iterations", ctypes.c_int),
                ("energy", ctypes.c_double), ("mp2", ctypes.c_double), ("conv", ctypes.c_double),
                ("t_submit", ctypes.c_double), ("t_admit", ctypes.c_double), ("t_done", ctypes.c_double),
                ("device_bytes", ctypes.c_int64), ("flops_per_iter", ctypes.c_double),
                ("peak_bytes", ctypes.c_int64), ("t_built", ctypes.c_double), ("message", ctypes.c_char * 160)]


_lib = None


def lib():
    """Load the shared library (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise CcsdError(-1, f"{LIB_PATH} is missing: run aquarius_b200.build.build()")
        L = ctypes.CDLL(str(LIB_PATH))
        vp, i32, i64, dbl = ctypes.c_void_p, ctypes.c_int32, ctypes.c_int64, ctypes.c_double
        P = ctypes.POINTER
        sig = {
            "ccsd_ctx_create": [ctypes.c_int, vp, P(vp)],
            "ccsd_ctx_destroy": [vp],
            "ccsd_ctx_synchronize": [vp],
            "ccsd_ctx_device_bytes": [vp, P(i64)],
            "ccsd_ctx_launch_count": [vp, P(i64)],
            "ccsd_ctx_plan_flops": [vp, P(dbl)],
            "ccsd_ctx_set_precision": [vp, ctypes.c_int, ctypes.c_int],
            "ccsd_ctx_set_profiling": [vp, ctypes.c_int],
            "ccsd_ctx_set_split_routing": [vp, ctypes.c_int],
            "ccsd_ctx_split_launches": [vp, P(i64)],
            "ccsd_server_options_default": [P(ServerOptions)],
            "ccsd_server_create": [P(ServerOptions), P(vp)],
            "ccsd_server_submit_synthetic": [vp, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_uint64, P(i64)],
            "ccsd_server_submit_factor": [vp, ctypes.c_int, vp, vp, ctypes.c_int, vp, vp, vp, P(i64)],
            "ccsd_server_poll": [vp, ctypes.c_int, P(ServerResult), P(ctypes.c_int)],
            "ccsd_server_wait": [vp, dbl],
            "ccsd_server_stats": [vp, P(ctypes.c_int), P(ctypes.c_int), P(i64), P(ctypes.c_int)],
            "ccsd_server_destroy": [vp],
            "ccsd_ctx_profile_report": [vp, ctypes.c_char_p, i64, P(i64)],
            "ccsd_ctx_set_spaces": [vp, ctypes.c_int, vp, vp, vp, vp],
            "ccsd_tensor_create": [vp, ctypes.c_char_p, vp, vp, ctypes.c_int, P(i32)],
            "ccsd_tensor_destroy": [vp, i32],
            "ccsd_tensor_ndim": [vp, i32, P(ctypes.c_int)],
            "ccsd_tensor_spin_cases": [vp, i32, P(ctypes.c_int), vp],
            "ccsd_tensor_block_size": [vp, i32, vp, vp, P(i64)],
            "ccsd_tensor_write_block": [vp, i32, vp, vp, vp],
            "ccsd_tensor_read_block": [vp, i32, vp, vp, vp],
            "ccsd_tensor_write": [vp, i32, vp, vp, i64, vp, vp, dbl, dbl],
            "ccsd_tensor_read": [vp, i32, vp, vp, i64, vp, vp],
            "ccsd_tensor_fill": [vp, i32, dbl],
            "ccsd_contract": [vp, dbl, i32, ctypes.c_char_p, i32, ctypes.c_char_p, dbl, i32, ctypes.c_char_p],
            "ccsd_sum": [vp, dbl, i32, ctypes.c_char_p, dbl, i32, ctypes.c_char_p],
            "ccsd_scale": [vp, i32, dbl],
            "ccsd_dot": [vp, i32, ctypes.c_char_p, i32, ctypes.c_char_p, P(dbl)],
            "ccsd_norm": [vp, i32, ctypes.c_int, P(dbl)],
            "ccsd_weight": [vp, i32, vp, vp, vp, vp, dbl],
            "ccsd_options_default": [P(Options)],
            "ccsd_hamiltonian_from_factor": [vp, ctypes.c_int, vp, vp, vp, ctypes.c_int, P(Hamiltonian)],
            "ccsd_hamiltonian_destroy": [vp, P(Hamiltonian)],
            "ccsd_hamiltonian_create": [vp, ctypes.c_int, P(Hamiltonian)],
            "ccsd_hamiltonian_from_integrals": [vp, ctypes.c_int, vp, vp, ctypes.c_int, P(Hamiltonian)],
            "ccsd_fcidump_read": [ctypes.c_char_p, ctypes.c_int, P(ctypes.c_int), P(ctypes.c_int), P(dbl), vp, vp],
            "ccsd_hamiltonian_from_fcidump": [vp, ctypes.c_char_p, ctypes.c_int, ctypes.c_int, P(Hamiltonian),
                                              P(dbl)],
            "ccsd_solver_create": [vp, P(Hamiltonian), P(Options), P(vp)],
            "ccsd_solver_destroy": [vp],
            "ccsd_diis_create": [vp, ctypes.c_int, ctypes.c_int, dbl, P(vp)],
            "ccsd_diis_extrapolate": [vp, ctypes.c_int, vp, vp, vp],
            "ccsd_diis_coefficients": [vp, P(ctypes.c_int), vp],
            "ccsd_diis_destroy": [vp],
            "ccsd_slice_choice": [ctypes.c_int, vp, dbl, vp],
            "ccsd_solver_slice_report": [vp, ctypes.c_char_p, i64, P(i64)],
            "ccsd_solver_mp2": [vp, P(dbl)],
            "ccsd_solver_iterate": [vp, P(dbl), P(dbl)],
            "ccsd_solver_iterate_async": [vp],
            "ccsd_solver_status": [vp, P(dbl), P(dbl), P(ctypes.c_int)],
            "ccsd_solver_run": [vp, P(dbl), P(dbl), P(ctypes.c_int)],
            "ccsd_solver_amplitudes": [vp, P(i32), P(i32)],
            "ccsd_solver_flops": [vp, P(dbl)],
            "ccsd_solver_mode": [vp, P(ctypes.c_int), P(ctypes.c_int)],
            "ccsd_plan_query": [ctypes.c_int, vp, vp, P(Options), ctypes.c_int, P(dbl), P(i64)],
            "ccsd_rhf_plan_query": [ctypes.c_int, vp, vp, P(Options), P(dbl), P(i64)],
            "ccsd_rhf_hamiltonian_from_factor": [vp, ctypes.c_int, vp, vp, vp, P(RHFHamiltonian)],
            "ccsd_rhf_hamiltonian_from_integrals": [vp, ctypes.c_int, vp, vp, P(RHFHamiltonian)],
            "ccsd_rhf_hamiltonian_destroy": [vp, P(RHFHamiltonian)],
            "ccsd_rhf_solver_create": [vp, P(RHFHamiltonian), P(Options), P(vp)],
            "ccsd_rhf_solver_hbar": [vp, P(RHFHbar)],
            "ccsd_solver_hbar": [vp, P(Hamiltonian)],
            "ccsd_ctx_plan_export": [vp, ctypes.c_char_p],
            "ccsd_plan_export_solver": [ctypes.c_int, ctypes.c_int, vp, vp, vp, vp, ctypes.c_int, ctypes.c_char_p],
            "ccsd_lambda_solver_create": [vp, P(Hamiltonian), vp, P(Options), P(vp)],
            "ccsd_lambda_plan_query": [ctypes.c_int, vp, vp, P(Options), P(dbl), P(dbl), P(i64)],
            "ccsd_hamiltonian_from_ao": [vp, ctypes.c_int, ctypes.c_int, ctypes.c_int, vp, vp, vp, ctypes.c_int,
                                         P(Hamiltonian), P(dbl)],
            "ccsd_rhf_hamiltonian_from_ao": [vp, ctypes.c_int, ctypes.c_int, ctypes.c_int, vp, vp, vp,
                                             P(RHFHamiltonian), P(dbl)],
            "ccsd_dot_batch_noalloc": [vp, vp, vp, ctypes.c_int, i64, vp],
            "ccsd_synth_irreps": [ctypes.c_uint64, ctypes.c_int, ctypes.c_int, ctypes.c_int, vp, vp, vp],
            "ccsd_synth_problem": [ctypes.c_uint64, ctypes.c_int, vp, vp, vp, vp, vp],
        }
        for name, args in sig.items():
            f = getattr(L, name)
            f.argtypes = args
            f.restype = None if name in ("ccsd_options_default", "ccsd_server_options_default") else ctypes.c_int
        L.ccsd_last_error.argtypes = [vp]
        L.ccsd_last_error.restype = ctypes.c_char_p
        _lib = L
    return _lib


def _ptr(a):
    return a.ctypes.data_as(ctypes.c_void_p) if a is not None else None


def _ints(xs):
    return np.ascontiguousarray(np.asarray(xs, dtype=np.int32))


def _check(code, ctx=None):
    if code != CCSD_OK:
        msg = lib().ccsd_last_error(ctx)
        raise CcsdError(code, (msg or b"").decode())


# ---------------------------------------------------------------------------
# synthetic inputs
# ---------------------------------------------------------------------------

def synth_irreps(seed: int, nirrep: int, o: int, v: int):
    occ = np.zeros(nirrep, np.int32)
    vrt = np.zeros(nirrep, np.int32)
    aux = np.zeros(nirrep, np.int32)
    _check(lib().ccsd_synth_irreps(seed, nirrep, o, v, _ptr(occ), _ptr(vrt), _ptr(aux)))
    return occ, vrt, aux


def synth_problem(seed: int, o: int, v: int, nirrep: int = 1, with_B: bool = True):
    """Seeded synthetic closed-shell problem: (eps[n], B[naux,n,n] or None, occ, vrt, aux irrep counts)."""
    if nirrep == 1:
        occ, vrt = np.array([o], np.int32), np.array([v], np.int32)
        aux = np.array([3 * (o + v)], np.int32)
    else:
        occ, vrt, aux = synth_irreps(seed, nirrep, o, v)
    n = o + v
    naux = int(aux.sum())
    eps = np.zeros(n)
    B = np.zeros((naux, n, n)) if with_B else None
    _check(lib().ccsd_synth_problem(seed, nirrep, _ptr(occ), _ptr(vrt), _ptr(aux), _ptr(eps), _ptr(B)))
    return eps, B, occ, vrt, aux


def dot_batch_noalloc(stream: int, x_ptr: int, y_ptrs, n: int, out_ptr: int):
    """out[j] = <x, y_j> on caller-owned device buffers; the library allocates nothing
    (see ccsd_dot_batch_noalloc in include/ccsd_b200.h).  Stream-ordered, no sync."""
    ys = (ctypes.c_void_p * max(len(y_ptrs), 1))(*[ctypes.c_void_p(p) for p in y_ptrs])
    _check(lib().ccsd_dot_batch_noalloc(ctypes.c_void_p(stream), ctypes.c_void_p(x_ptr), ys, len(y_ptrs), n,
                                        ctypes.c_void_p(out_ptr)))


def plan_query(vrt, occ, diis_order=8, pack_vvvv=True, precision="fp64"):
    """Host-only planning: (algorithmic FP64 flops per iteration, device bytes of a solve)."""
    vrt, occ = _ints(vrt), _ints(occ)
    o = Options()
    lib().ccsd_options_default(ctypes.byref(o))
    o.diis_order = diis_order
    o.precision = PREC[precision]
    fl, by = ctypes.c_double(), ctypes.c_int64()
    _check(lib().ccsd_plan_query(len(vrt), _ptr(vrt), _ptr(occ), ctypes.byref(o), 1 if pack_vvvv else 0,
                                 ctypes.byref(fl), ctypes.byref(by)))
    return fl.value, by.value


def lambda_plan_query(vrt, occ, diis_order=8, precision="fp64"):
    """Host-only planning of CCSD + Hbar + Lambda-CCSD (unpacked <ab||ef>): (flops of forming
    Hbar, flops per Lambda iteration, peak device bytes)."""
    vrt, occ = _ints(vrt), _ints(occ)
    o = Options()
    lib().ccsd_options_default(ctypes.byref(o))
    o.diis_order = diis_order
    o.precision = PREC[precision]
    hf, fl, by = ctypes.c_double(), ctypes.c_double(), ctypes.c_int64()
    _check(lib().ccsd_lambda_plan_query(len(vrt), _ptr(vrt), _ptr(occ), ctypes.byref(o), ctypes.byref(hf),
                                        ctypes.byref(fl), ctypes.byref(by)))
    return hf.value, fl.value, by.value


METHODS = {"ccsd": 0, "rhf": 1, "lambda": 2}
PLANS = {"iteration": 0, "hbar": 1, "energy": 2}


def plan_export_solver(method, vrt, occ, which, path, vrt_beta=None, occ_beta=None):
    """Host-only: write one recorded plan of a CCSD / RHF / Lambda solver for these sizes
    (ccsd_plan_export_solver), for replay by a host-side checker."""
    vrt, occ = _ints(vrt), _ints(occ)
    vb = _ints(vrt_beta) if vrt_beta is not None else None
    ob = _ints(occ_beta) if occ_beta is not None else None
    _check(lib().ccsd_plan_export_solver(METHODS[method], len(vrt), _ptr(vrt), _ptr(occ),
                                         _ptr(vb) if vb is not None else None, _ptr(ob) if ob is not None else None,
                                         PLANS[which], str(path).encode()))


def rhf_plan_query(vrt, occ, diis_order=8, precision="fp64", refine_tol=0.0):
    """Host-only planning of the closed-shell iteration: (flops per iteration, device bytes)."""
    vrt, occ = _ints(vrt), _ints(occ)
    o = Options()
    lib().ccsd_options_default(ctypes.byref(o))
    o.diis_order = diis_order
    o.precision = PREC[precision]
    o.refine_tol = refine_tol
    fl, by = ctypes.c_double(), ctypes.c_int64()
    _check(lib().ccsd_rhf_plan_query(len(vrt), _ptr(vrt), _ptr(occ), ctypes.byref(o), ctypes.byref(fl),
                                     ctypes.byref(by)))
    return fl.value, by.value


FCIDUMP_FULL_FOCK = 1
FCIDUMP_SEMICANONICAL = 2


def fcidump_read(path, full_fock=False):
    """Parse an FCIDUMP on the host (ccsd_fcidump_read): dict with norb, nelec, ecore,
    h (n x n) and eri (n^4, (pq|rs) with all eight images)."""
    flags = FCIDUMP_FULL_FOCK if full_fock else 0
    norb, nelec, ecore = ctypes.c_int(), ctypes.c_int(), ctypes.c_double()
    p = os.fsencode(path)
    _check(lib().ccsd_fcidump_read(p, flags, ctypes.byref(norb), ctypes.byref(nelec), ctypes.byref(ecore), None,
                                   None))
    n = norb.value
    h = np.zeros((n, n))
    eri = np.zeros((n, n, n, n))
    _check(lib().ccsd_fcidump_read(p, flags, ctypes.byref(norb), ctypes.byref(nelec), ctypes.byref(ecore), _ptr(h),
                                   _ptr(eri)))
    return {"norb": n, "nelec": nelec.value, "ecore": ecore.value, "h": h, "eri": eri}


# ---------------------------------------------------------------------------
# context / tensors
# ---------------------------------------------------------------------------

class Tensor:
    def __init__(self, ctx: "Context", handle: int, name: str, nout, nin, packed=False, plain=False):
        self.ctx, self.h, self.name, self.packed, self.plain = ctx, handle, name, packed, plain
        self.nout, self.nin = tuple(nout), tuple(nin)
        self.group = [0] * nout[0] + [1] * nout[1] + [2] * nin[0] + [3] * nin[1]
        self.ndim = len(self.group)

    def spin_cases(self):
        n = ctypes.c_int()
        _check(lib().ccsd_tensor_spin_cases(self.ctx.c, self.h, ctypes.byref(n), None), self.ctx.c)
        a = np.zeros(4 * n.value, np.int32)
        _check(lib().ccsd_tensor_spin_cases(self.ctx.c, self.h, ctypes.byref(n), _ptr(a)), self.ctx.c)
        return [tuple(a[4 * i:4 * i + 4]) for i in range(n.value)]

    def case_spins(self, alpha):
        """spin (0 alpha, 1 beta) of every position for a spin case."""
        gs = [self.nout[0], self.nout[1], self.nin[0], self.nin[1]]
        out = []
        for g in range(4):
            out += [0] * alpha[g] + [1] * (gs[g] - alpha[g])
        return out

    def block_size(self, alpha, irreps=None):
        n = ctypes.c_int64()
        irr = _ints(irreps if irreps is not None else [0] * self.ndim)
        _check(lib().ccsd_tensor_block_size(self.ctx.c, self.h, _ptr(_ints(alpha)), _ptr(irr), ctypes.byref(n)),
               self.ctx.c)
        return n.value

    def block_shape(self, alpha, irreps=None):
        irreps = irreps if irreps is not None else [0] * self.ndim
        sp = self.case_spins(alpha)
        return tuple(self.ctx.count(self.group[p] % 2, sp[p], irreps[p]) for p in range(self.ndim))

    def read_block(self, alpha, irreps=None):
        n = self.block_size(alpha, irreps)
        out = np.zeros(max(n, 1))
        irr = _ints(irreps if irreps is not None else [0] * self.ndim)
        _check(lib().ccsd_tensor_read_block(self.ctx.c, self.h, _ptr(_ints(alpha)), _ptr(irr), _ptr(out)), self.ctx.c)
        return out[:n]

    def write_block(self, alpha, data, irreps=None):
        data = np.ascontiguousarray(np.asarray(data, dtype=np.float64).reshape(-1, order="F"))
        irr = _ints(irreps if irreps is not None else [0] * self.ndim)
        _check(lib().ccsd_tensor_write_block(self.ctx.c, self.h, _ptr(_ints(alpha)), _ptr(irr), _ptr(data)),
               self.ctx.c)

    def write(self, alpha, keys, vals, a=1.0, b=0.0, irreps=None):
        keys = np.ascontiguousarray(np.asarray(keys, dtype=np.int64))
        vals = np.ascontiguousarray(np.asarray(vals, dtype=np.float64))
        irr = _ints(irreps if irreps is not None else [0] * self.ndim)
        _check(lib().ccsd_tensor_write(self.ctx.c, self.h, _ptr(_ints(alpha)), _ptr(irr), len(keys), _ptr(keys),
                                       _ptr(vals), a, b), self.ctx.c)

    def read(self, alpha, keys, irreps=None):
        keys = np.ascontiguousarray(np.asarray(keys, dtype=np.int64))
        vals = np.zeros(len(keys))
        irr = _ints(irreps if irreps is not None else [0] * self.ndim)
        _check(lib().ccsd_tensor_read(self.ctx.c, self.h, _ptr(_ints(alpha)), _ptr(irr), len(keys), _ptr(keys),
                                      _ptr(vals)), self.ctx.c)
        return vals

    def fill(self, val):
        _check(lib().ccsd_tensor_fill(self.ctx.c, self.h, float(val)), self.ctx.c)

    def elements(self):
        """stored elements over every spin case and irrep block"""
        n = 0
        for alpha in self.spin_cases():
            for irr in itertools.product(range(self.ctx.nirrep), repeat=self.ndim):
                x = 0
                for h in irr:
                    x ^= h
                if not x:
                    n += self.block_size(alpha, irr)
        return n

    def norm(self, p=0):
        out = ctypes.c_double()
        _check(lib().ccsd_norm(self.ctx.c, self.h, p, ctypes.byref(out)), self.ctx.c)
        return out.value

    def __getitem__(self, idx):
        return _Indexed(self, idx, 1.0)

    def __setitem__(self, idx, expr):
        if isinstance(expr, _Assign):      # produced by += / -= on an _Indexed
            return
        _assign(self, idx, expr, beta=0.0)

    # -- full spin-orbital array (tests) -------------------------------------------------
    def to_full(self):
        """Dense full spin-orbital array: every index runs over [alpha | beta] of its space,
        irrep-major inside a spin; antisymmetric images inside groups are filled in.
        A plain tensor gives its spatial array (irrep-major per index)."""
        ctx = self.ctx
        if self.plain:
            full = np.zeros([ctx.total(self.group[p] % 2) for p in range(self.ndim)])
            alpha = self.spin_cases()[0]
            for irr in itertools.product(range(ctx.nirrep), repeat=self.ndim):
                x = 0
                for h in irr:
                    x ^= h
                if x or self.block_size(alpha, irr) == 0:
                    continue
                shape = self.block_shape(alpha, irr)
                sl = tuple(slice(ctx.offset(self.group[p] % 2, irr[p]), ctx.offset(self.group[p] % 2, irr[p]) + shape[p])
                           for p in range(self.ndim))
                full[sl] = self.read_block(alpha, irr).reshape(shape, order="F")
            return full
        dims = []
        for p in range(self.ndim):
            sp = self.group[p] % 2
            dims.append(ctx.total(sp, 0) + ctx.total(sp, 1))
        full = np.zeros(dims)
        groups = [[p for p in range(self.ndim) if self.group[p] == g] for g in range(4)]
        for alpha in self.spin_cases():
            spins = self.case_spins(alpha)
            for irr in itertools.product(range(ctx.nirrep), repeat=self.ndim):
                x = 0
                for h in irr:
                    x ^= h
                if x:
                    continue
                if self.block_size(alpha, irr) == 0:
                    continue
                shape = self.block_shape(alpha, irr)
                blk = self.read_block(alpha, irr).reshape(shape, order="F")
                perms = [list(itertools.permutations(gp)) for gp in groups]
                for combo in itertools.product(*perms):
                    perm = list(range(self.ndim))
                    for gp, pg in zip(groups, combo):
                        for a_, b_ in zip(gp, pg):
                            perm[a_] = b_
                    sign = 1
                    pp = list(perm)
                    for i in range(len(pp)):
                        while pp[i] != i:
                            j = pp[i]
                            pp[i], pp[j] = pp[j], pp[i]
                            sign = -sign
                    # position q of the image takes original position perm[q]
                    sl = []
                    for q in range(self.ndim):
                        p0 = perm[q]
                        sp = self.group[p0] % 2
                        lo = ctx.spin_start(sp, spins[p0]) + ctx.offset(sp, irr[p0], spins[p0])
                        sl.append(slice(lo, lo + shape[p0]))
                    full[tuple(sl)] = sign * np.transpose(blk, perm)
        return full


class _Indexed:
    def __init__(self, t, idx, f):
        self.t, self.idx, self.f = t, idx, f

    def __mul__(self, other):
        if isinstance(other, _Indexed):
            return _Mult(self, other, self.f * other.f)
        return _Indexed(self.t, self.idx, self.f * other)

    def __rmul__(self, f):
        return _Indexed(self.t, self.idx, self.f * f)

    def __iadd__(self, expr):
        _assign(self.t, self.idx, expr, beta=1.0)
        return _Assign()

    def __isub__(self, expr):
        _assign(self.t, self.idx, -1.0 * expr, beta=1.0)
        return _Assign()


class _Mult:
    def __init__(self, a, b, f):
        self.a, self.b, self.f = a, b, f

    def __rmul__(self, f):
        return _Mult(self.a, self.b, self.f * f)


class _Assign:
    pass


def _assign(t, idx, expr, beta):
    ctx = t.ctx
    if isinstance(expr, _Mult):
        ctx.contract(expr.f, expr.a.t, expr.a.idx, expr.b.t, expr.b.idx, beta, t, idx)
    elif isinstance(expr, _Indexed):
        ctx.sum(expr.f, expr.t, expr.idx, beta, t, idx)
    else:
        raise TypeError("unsupported expression")


class Context:
    """device < 0: a planning-only context (no GPU): statements plan and account bytes and
    flops, nothing runs, tensor data cannot be read or written."""

    def __init__(self, device: int = 0, stream: int | None = None):
        c = ctypes.c_void_p()
        _check(lib().ccsd_ctx_create(device, stream, ctypes.byref(c)))
        self.c = c
        self.nirrep = 1
        self._counts = None

    def close(self):
        if self.c:
            _check(lib().ccsd_ctx_destroy(self.c))
            self.c = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def set_spaces(self, vrt, occ, vrt_beta=None, occ_beta=None):
        vrt, occ = _ints(vrt), _ints(occ)
        vb = _ints(vrt_beta if vrt_beta is not None else vrt)
        ob = _ints(occ_beta if occ_beta is not None else occ)
        self.nirrep = len(vrt)
        _check(lib().ccsd_ctx_set_spaces(self.c, self.nirrep, _ptr(vrt), _ptr(vb), _ptr(occ), _ptr(ob)), self.c)
        self._counts = {(0, 0): vrt, (0, 1): vb, (1, 0): occ, (1, 1): ob}

    def count(self, space, spin, irrep):
        return int(self._counts[(space, spin)][irrep])

    def total(self, space, spin=0):
        return int(self._counts[(space, spin)].sum())

    def offset(self, space, irrep, spin=0):
        return int(self._counts[(space, spin)][:irrep].sum())

    def spin_start(self, space, spin):
        """first full spin-orbital index of a spin inside a space ([alpha | beta])"""
        return 0 if spin == 0 else self.total(space, 0)

    def set_precision(self, precision="fp64", slices=0):
        _check(lib().ccsd_ctx_set_precision(self.c, PREC[precision], slices), self.c)

    def set_split_routing(self, mode="auto"):
        """"auto": size thresholds keep small products on FP64; "all": every product split."""
        _check(lib().ccsd_ctx_set_split_routing(self.c, {"auto": 0, "all": 1}[mode]), self.c)

    def split_launches(self):
        n = ctypes.c_int64()
        _check(lib().ccsd_ctx_split_launches(self.c, ctypes.byref(n)), self.c)
        return n.value

    def tensor(self, name, nout, nin, packed=False, plain=False):
        """plain: a spatial tensor without antisymmetry or spin cases (closed-shell forms)"""
        h = ctypes.c_int32()
        flags = (TENSOR_PACKED if packed else 0) | (TENSOR_PLAIN if plain else 0)
        _check(lib().ccsd_tensor_create(self.c, name.encode(), _ptr(_ints(nout)), _ptr(_ints(nin)), flags,
                                        ctypes.byref(h)), self.c)
        return Tensor(self, h.value, name, nout, nin, packed, plain)

    def contract(self, alpha, A, ia, B, ib, beta, C, ic):
        _check(lib().ccsd_contract(self.c, alpha, A.h, ia.encode(), B.h, ib.encode(), beta, C.h, ic.encode()), self.c)

    def sum(self, alpha, A, ia, beta, B, ib):
        _check(lib().ccsd_sum(self.c, alpha, A.h, ia.encode(), beta, B.h, ib.encode()), self.c)

    def dot(self, A, ia, B, ib):
        out = ctypes.c_double()
        _check(lib().ccsd_dot(self.c, A.h, ia.encode(), B.h, ib.encode(), ctypes.byref(out)), self.c)
        return out.value

    def scale(self, A, alpha):
        _check(lib().ccsd_scale(self.c, A.h, alpha), self.c)

    def weight(self, A, dvrt, docc, dvrt_b=None, docc_b=None, shift=0.0):
        dv = np.ascontiguousarray(dvrt, dtype=np.float64)
        do = np.ascontiguousarray(docc, dtype=np.float64)
        dvb = np.ascontiguousarray(dvrt_b if dvrt_b is not None else dv, dtype=np.float64)
        dob = np.ascontiguousarray(docc_b if docc_b is not None else do, dtype=np.float64)
        _check(lib().ccsd_weight(self.c, A.h, _ptr(dv), _ptr(dvb), _ptr(do), _ptr(dob), shift), self.c)

    def synchronize(self):
        _check(lib().ccsd_ctx_synchronize(self.c), self.c)

    def device_bytes(self):
        n = ctypes.c_int64()
        _check(lib().ccsd_ctx_device_bytes(self.c, ctypes.byref(n)), self.c)
        return n.value

    def set_profiling(self, on=True):
        _check(lib().ccsd_ctx_set_profiling(self.c, 1 if on else 0), self.c)

    def profile_report(self):
        """{statement: {"launches", "ms", "flops"}} for the contraction kernels timed since
        profiling was enabled (clears the totals)."""
        import json
        need = ctypes.c_int64()
        _check(lib().ccsd_ctx_profile_report(self.c, None, 0, ctypes.byref(need)), self.c)
        buf = ctypes.create_string_buffer(int(need.value) + 16)
        _check(lib().ccsd_ctx_profile_report(self.c, buf, len(buf), ctypes.byref(need)), self.c)
        return json.loads(buf.value.decode())

    def plan_flops(self):
        """algorithmic flops of the last contraction statement (planner count)"""
        x = ctypes.c_double()
        _check(lib().ccsd_ctx_plan_flops(self.c, ctypes.byref(x)), self.c)
        return x.value

    def plan_export(self, path):
        """write the plan of the last contraction / sum statement as text (ccsd_ctx_plan_export)"""
        _check(lib().ccsd_ctx_plan_export(self.c, str(path).encode()), self.c)

    def launch_count(self):
        n = ctypes.c_int64()
        _check(lib().ccsd_ctx_launch_count(self.c, ctypes.byref(n)), self.c)
        return n.value

    def hamiltonian(self, pack_vvvv=False):
        """The 13 H blocks, zero-filled, for the caller to write (ccsd_hamiltonian_create)."""
        H = Hamiltonian()
        _check(lib().ccsd_hamiltonian_create(self.c, 1 if pack_vvvv else 0, ctypes.byref(H)), self.c)
        return HamiltonianHandle(self, H, pack_vvvv)

    def hamiltonian_from_integrals(self, fock, eri, pack_vvvv=True):
        """Closed-shell H from a spatial Fock matrix and dense (pq|rs) (occupied first)."""
        fock = np.ascontiguousarray(fock, dtype=np.float64)
        eri = np.ascontiguousarray(eri, dtype=np.float64)
        n = fock.shape[0]
        if fock.shape != (n, n) or eri.shape != (n, n, n, n):
            raise ValueError("fock must be (n, n) and eri (n, n, n, n)")
        H = Hamiltonian()
        _check(lib().ccsd_hamiltonian_from_integrals(self.c, n, _ptr(fock), _ptr(eri), 1 if pack_vvvv else 0,
                                                     ctypes.byref(H)), self.c)
        return HamiltonianHandle(self, H, pack_vvvv)

    def hamiltonian_from_fcidump(self, path, semicanonical=False, full_fock=False, pack_vvvv=True):
        """Read an FCIDUMP, set C1 closed-shell spaces and build H: (handle, E(SCF))."""
        flags = (FCIDUMP_SEMICANONICAL if semicanonical else 0) | (FCIDUMP_FULL_FOCK if full_fock else 0)
        H = Hamiltonian()
        escf = ctypes.c_double()
        _check(lib().ccsd_hamiltonian_from_fcidump(self.c, os.fsencode(path), flags, 1 if pack_vvvv else 0,
                                                   ctypes.byref(H), ctypes.byref(escf)), self.c)
        norb = ctypes.c_int()
        nelec = ctypes.c_int()
        _check(lib().ccsd_fcidump_read(os.fsencode(path), flags, ctypes.byref(norb), ctypes.byref(nelec), None, None,
                                       None))
        no = nelec.value // 2
        self.nirrep = 1
        self._counts = {(0, 0): _ints([norb.value - no]), (0, 1): _ints([norb.value - no]), (1, 0): _ints([no]),
                        (1, 1): _ints([no])}
        return HamiltonianHandle(self, H, pack_vvvv), escf.value

    def hamiltonian_from_factor(self, B, eps, aux_per_irrep=None, pack_vvvv=True):
        B = np.ascontiguousarray(B, dtype=np.float64)
        eps = np.ascontiguousarray(eps, dtype=np.float64)
        H = Hamiltonian()
        aux = _ints(aux_per_irrep) if aux_per_irrep is not None else None
        _check(lib().ccsd_hamiltonian_from_factor(self.c, B.shape[0], _ptr(B), _ptr(eps), _ptr(aux),
                                                  1 if pack_vvvv else 0, ctypes.byref(H)), self.c)
        return HamiltonianHandle(self, H, pack_vvvv)

    def rhf_hamiltonian_from_factor(self, B, eps, aux_per_irrep=None):
        """Closed-shell spatial blocks <pq|rs> from the factor B[P,p,q] and orbital energies."""
        B = np.ascontiguousarray(B, dtype=np.float64)
        eps = np.ascontiguousarray(eps, dtype=np.float64)
        H = RHFHamiltonian()
        aux = _ints(aux_per_irrep) if aux_per_irrep is not None else None
        _check(lib().ccsd_rhf_hamiltonian_from_factor(self.c, B.shape[0], _ptr(B), _ptr(eps), _ptr(aux),
                                                      ctypes.byref(H)), self.c)
        return RHFHamiltonianHandle(self, H)

    def rhf_hamiltonian_from_integrals(self, fock, eri):
        """Closed-shell spatial blocks from a Fock matrix and dense (pq|rs) (occupied first)."""
        fock = np.ascontiguousarray(fock, dtype=np.float64)
        eri = np.ascontiguousarray(eri, dtype=np.float64)
        n = fock.shape[0]
        if fock.shape != (n, n) or eri.shape != (n, n, n, n):
            raise ValueError("fock must be (n, n) and eri (n, n, n, n)")
        H = RHFHamiltonian()
        _check(lib().ccsd_rhf_hamiltonian_from_integrals(self.c, n, _ptr(fock), _ptr(eri), ctypes.byref(H)), self.c)
        return RHFHamiltonianHandle(self, H)

    def _ao_args(self, hcore, eri_ao, C, nocc):
        hcore = np.ascontiguousarray(hcore, dtype=np.float64)
        eri_ao = np.ascontiguousarray(eri_ao, dtype=np.float64)
        C = np.ascontiguousarray(C, dtype=np.float64)
        nao, nmo = C.shape
        if hcore.shape != (nao, nao) or eri_ao.shape != (nao, nao, nao, nao):
            raise ValueError("hcore must be (nao, nao), eri_ao (nao,)*4 and C (nao, nmo)")
        self.nirrep = 1
        self._counts = {(0, 0): _ints([nmo - nocc]), (0, 1): _ints([nmo - nocc]), (1, 0): _ints([nocc]),
                        (1, 1): _ints([nocc])}
        return hcore, eri_ao, C, nao, nmo

    def hamiltonian_from_ao(self, hcore, eri_ao, C, nocc, pack_vvvv=True):
        """Closed-shell H from AO quantities; the MO integrals are formed on the device.
        Returns (handle, SCF electronic energy of C)."""
        hcore, eri_ao, C, nao, nmo = self._ao_args(hcore, eri_ao, C, nocc)
        H = Hamiltonian()
        e = ctypes.c_double()
        _check(lib().ccsd_hamiltonian_from_ao(self.c, nao, nmo, nocc, _ptr(hcore), _ptr(eri_ao), _ptr(C),
                                              1 if pack_vvvv else 0, ctypes.byref(H), ctypes.byref(e)), self.c)
        return HamiltonianHandle(self, H, pack_vvvv), e.value

    def rhf_hamiltonian_from_ao(self, hcore, eri_ao, C, nocc):
        """Closed-shell spatial blocks from AO quantities (MO integrals formed on the device)."""
        hcore, eri_ao, C, nao, nmo = self._ao_args(hcore, eri_ao, C, nocc)
        H = RHFHamiltonian()
        e = ctypes.c_double()
        _check(lib().ccsd_rhf_hamiltonian_from_ao(self.c, nao, nmo, nocc, _ptr(hcore), _ptr(eri_ao), _ptr(C),
                                                  ctypes.byref(H), ctypes.byref(e)), self.c)
        return RHFHamiltonianHandle(self, H), e.value

    def solver(self, H, **kw):
        return Solver(self, H, **kw)

    def diis(self, order=5, start=1, damping=0.0):
        """DIIS over caller tensors (ccsd_diis_*), the reference's DIIS<T>."""
        return Diis(self, order, start, damping)


class Diis:
    """DIIS<T>::extrapolate (src/convergence/diis.hpp:70-227) on the device over engine
    tensors: extrapolate([T1, T2], [Z1, Z2]) overwrites both lists with the combinations."""

    def __init__(self, ctx, order, start, damping):
        self.ctx, self.order = ctx, order
        d = ctypes.c_void_p()
        _check(lib().ccsd_diis_create(ctx.c, order, start, float(damping), ctypes.byref(d)), ctx.c)
        self.d = d

    def extrapolate(self, x, dx, weights=None):
        n = len(x)
        xa = np.array([t.h for t in x], dtype=np.int32)
        da = np.array([t.h for t in dx], dtype=np.int32)
        w = None if weights is None else np.ascontiguousarray(np.asarray(weights, dtype=np.float64))
        _check(lib().ccsd_diis_extrapolate(self.d, n, _ptr(xa), _ptr(da), None if w is None else _ptr(w)),
               self.ctx.c)

    def coefficients(self):
        """(stored pairs, coefficients by age: c[0] for the pair just stored)"""
        n = ctypes.c_int()
        c = np.zeros(max(self.order, 1))
        _check(lib().ccsd_diis_coefficients(self.d, ctypes.byref(n), _ptr(c)), self.ctx.c)
        return n.value, c

    def close(self):
        if self.d:
            _check(lib().ccsd_diis_destroy(self.d), self.ctx.c)
            self.d = None


class HamiltonianHandle:
    def __init__(self, ctx, H, packed):
        self.ctx, self.H = ctx, H
        self.tensors = {f: Tensor(ctx, getattr(H, f), f, *H_SHAPES[f], packed=(packed and f == "VABEF"))
                        for f in H_FIELDS}

    def __getitem__(self, name):
        return self.tensors[name]

    def destroy(self):
        if self.ctx.c:
            _check(lib().ccsd_hamiltonian_destroy(self.ctx.c, ctypes.byref(self.H)), self.ctx.c)


class RHFHamiltonianHandle:
    def __init__(self, ctx, H):
        self.ctx, self.H = ctx, H
        self.tensors = {f: Tensor(ctx, getattr(H, f), f, *RHF_SHAPES[f], plain=True) for f in RHF_FIELDS}

    def __getitem__(self, name):
        return self.tensors[name]

    def destroy(self):
        if self.ctx.c:
            _check(lib().ccsd_rhf_hamiltonian_destroy(self.ctx.c, ctypes.byref(self.H)), self.ctx.c)


def _options(conv_tol=1e-9, max_iter=50, diis_order=5, diis_start=1, precision="fp64", slices=0,
             use_graph=False, refine_tol=0.0, autotune_de=0.0):
    o = Options()
    lib().ccsd_options_default(ctypes.byref(o))
    o.conv_tol, o.max_iter, o.diis_order, o.diis_start = conv_tol, max_iter, diis_order, diis_start
    o.precision, o.slices, o.use_graph = PREC[precision], slices, 1 if use_graph else 0
    o.refine_tol = refine_tol
    o.autotune_de = autotune_de
    return o


def slice_choice(dE, budget):
    """The slice autotuner's rule (ccsd_slice_choice): which statements take one slice fewer."""
    d = np.ascontiguousarray(np.asarray(dE, dtype=np.float64))
    out = np.zeros(len(d), np.int32)
    _check(lib().ccsd_slice_choice(len(d), _ptr(d), float(budget), _ptr(out)))
    return out.astype(bool)


class HbarHandle:
    """Spin-orbital Hbar blocks (ccsd_solver_hbar), keyed like the H blocks; owned by the
    CCSD solver that formed them."""

    def __init__(self, ctx, H):
        self.ctx, self.H = ctx, H
        self.tensors = {f: Tensor(ctx, getattr(H, f), f, *H_SHAPES[f]) for f in H_FIELDS}

    def __getitem__(self, name):
        return self.tensors[name]


class Solver:
    """CCSD solver over a spin-orbital H (CCSD) or a closed-shell spatial H (RHFCCSD)."""

    def __init__(self, ctx, H, **kw):
        self.ctx = ctx
        o = _options(**kw)
        s = ctypes.c_void_p()
        self.rhf = isinstance(H, RHFHamiltonianHandle)
        create = lib().ccsd_rhf_solver_create if self.rhf else lib().ccsd_solver_create
        _check(create(ctx.c, ctypes.byref(H.H), ctypes.byref(o), ctypes.byref(s)), ctx.c)
        self.s = s
        self._amplitudes(((1, 0), (0, 1)), ((2, 0), (0, 2)), "T")

    def _amplitudes(self, shape1, shape2, name):
        t1, t2 = ctypes.c_int32(), ctypes.c_int32()
        _check(lib().ccsd_solver_amplitudes(self.s, ctypes.byref(t1), ctypes.byref(t2)), self.ctx.c)
        self.T1 = Tensor(self.ctx, t1.value, name + "1", *shape1, plain=self.rhf)
        self.T2 = Tensor(self.ctx, t2.value, name + "2", *shape2, plain=self.rhf)

    def close(self):
        if self.s:
            _check(lib().ccsd_solver_destroy(self.s), self.ctx.c)
            self.s = None

    @property
    def mp2(self):
        x = ctypes.c_double()
        _check(lib().ccsd_solver_mp2(self.s, ctypes.byref(x)), self.ctx.c)
        return x.value

    def iterate(self):
        e, c = ctypes.c_double(), ctypes.c_double()
        _check(lib().ccsd_solver_iterate(self.s, ctypes.byref(e), ctypes.byref(c)), self.ctx.c)
        return e.value, c.value

    def slice_report(self):
        """[(slices, measured dE, statement label)] of the split statements (the autotuner's
        choice once it has run)."""
        need = ctypes.c_int64()
        _check(lib().ccsd_solver_slice_report(self.s, None, 0, ctypes.byref(need)), self.ctx.c)
        buf = ctypes.create_string_buffer(max(need.value, 1))
        _check(lib().ccsd_solver_slice_report(self.s, buf, need.value, ctypes.byref(need)), self.ctx.c)
        out = []
        for line in buf.value.decode().splitlines():
            ns, de, label = line.split("\t", 2)
            out.append((int(ns), float(de), label))
        return out

    def iterate_async(self):
        _check(lib().ccsd_solver_iterate_async(self.s), self.ctx.c)

    def status(self):
        e, c, i = ctypes.c_double(), ctypes.c_double(), ctypes.c_int()
        _check(lib().ccsd_solver_status(self.s, ctypes.byref(e), ctypes.byref(c), ctypes.byref(i)), self.ctx.c)
        return e.value, c.value, i.value

    def run(self):
        e, c, i = ctypes.c_double(), ctypes.c_double(), ctypes.c_int()
        code = lib().ccsd_solver_run(self.s, ctypes.byref(e), ctypes.byref(c), ctypes.byref(i))
        if code not in (CCSD_OK, 6):
            _check(code, self.ctx.c)
        return e.value, c.value, i.value

    def mode(self):
        """contraction mode of the next iteration: "fp64", "split3", "split4" (BF16 slices) or
        "i8split3" .. "i8split5" (INT8 slices)"""
        p, n = ctypes.c_int(), ctypes.c_int()
        _check(lib().ccsd_solver_mode(self.s, ctypes.byref(p), ctypes.byref(n)), self.ctx.c)
        return "fp64" if p.value == 0 else (f"split{n.value}" if p.value == 1 else f"i8split{n.value}")

    def flops(self):
        x = ctypes.c_double()
        _check(lib().ccsd_solver_flops(self.s, ctypes.byref(x)), self.ctx.c)
        return x.value

    def hbar(self):
        """Hbar from the current amplitudes, as tensors owned by the solver.  Closed-shell
        solver: dict of the RHF intermediates (rhfccsd.cxx:110-186).  Spin-orbital solver: an
        HbarHandle with the 13 blocks of STTwoElectronOperator(H, T, isHbar)."""
        if not self.rhf:
            h = Hamiltonian()
            _check(lib().ccsd_solver_hbar(self.s, ctypes.byref(h)), self.ctx.c)
            return HbarHandle(self.ctx, h)
        h = RHFHbar()
        _check(lib().ccsd_rhf_solver_hbar(self.s, ctypes.byref(h)), self.ctx.c)
        return {f: Tensor(self.ctx, getattr(h, f), f, *HBAR_SHAPES[f], plain=True) for f in HBAR_SHAPES}

    def lambda_solver(self, hbar=None, **kw):
        """Lambda-CCSD on `hbar` (default: this solver's Hbar, formed now) and this solver's T."""
        return LambdaSolver(self, self.hbar() if hbar is None else hbar, **kw)


class LambdaSolver(Solver):
    """Lambda-CCSD (LambdaCCSD, lambdaccsd.cxx) on an Hbar and a spin-orbital CCSD solver's
    amplitudes.  L1 is [i, a] and L2 [i, j, a, b]; energy() is 1/4 <mn||ef> l_mn^ef."""

    def __init__(self, ccsd, hbar, **kw):
        self.ctx, self.rhf = ccsd.ctx, False
        self.ccsd, self.hbar_blocks = ccsd, hbar
        o = _options(**kw)
        s = ctypes.c_void_p()
        _check(lib().ccsd_lambda_solver_create(self.ctx.c, ctypes.byref(hbar.H), ccsd.s, ctypes.byref(o),
                                               ctypes.byref(s)), self.ctx.c)
        self.s = s
        self._amplitudes(((0, 1), (1, 0)), ((0, 2), (2, 0)), "L")
        self.L1, self.L2 = self.T1, self.T2

    def hbar(self):
        raise CcsdError(9, "a Lambda solver forms no Hbar")


class Server:
    """Continuous batching of solves on one device (ccsd_server_*): submit requests as
    they arrive, poll finished results; admission by planned device bytes."""

    def __init__(self, device=0, memory_budget=0, max_active=16, pack_vvvv=True, precision="fp64", conv_tol=1e-9,
                 max_iter=100, diis_order=8, diis_start=1, refine_tol=0.0, use_graph=False):
        o = ServerOptions()
        lib().ccsd_server_options_default(ctypes.byref(o))
        o.device, o.memory_budget, o.max_active, o.pack_vvvv = device, int(memory_budget), max_active, int(pack_vvvv)
        o.solve.precision, o.solve.conv_tol, o.solve.max_iter = PREC[precision], conv_tol, max_iter
        o.solve.diis_order, o.solve.diis_start, o.solve.refine_tol = diis_order, diis_start, refine_tol
        o.solve.use_graph = 1 if use_graph else 0
        s = ctypes.c_void_p()
        _check(lib().ccsd_server_create(ctypes.byref(o), ctypes.byref(s)))
        self.s = s

    def submit_synthetic(self, o, v, nirrep=1, seed=0):
        i = ctypes.c_int64()
        _check(lib().ccsd_server_submit_synthetic(self.s, nirrep, o, v, seed, ctypes.byref(i)))
        return i.value

    def submit_factor(self, B, eps, vrt, occ, aux_per_irrep=None):
        B = np.ascontiguousarray(B, dtype=np.float64)
        eps = np.ascontiguousarray(eps, dtype=np.float64)
        vrt, occ = _ints(vrt), _ints(occ)
        aux = _ints(aux_per_irrep) if aux_per_irrep is not None else None
        i = ctypes.c_int64()
        _check(lib().ccsd_server_submit_factor(self.s, len(vrt), _ptr(vrt), _ptr(occ), B.shape[0], _ptr(B), _ptr(eps),
                                               _ptr(aux), ctypes.byref(i)))
        return i.value

    def poll(self, max_results=256):
        buf = (ServerResult * max_results)()
        n = ctypes.c_int()
        _check(lib().ccsd_server_poll(self.s, max_results, buf, ctypes.byref(n)))
        out = [{f: getattr(buf[k], f) for f, _ in ServerResult._fields_} for k in range(n.value)]
        for r in out:
            r["message"] = r["message"].decode(errors="replace")
        return out

    def wait(self, timeout=3600.0):
        _check(lib().ccsd_server_wait(self.s, timeout))

    def stats(self):
        q, a, pa = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        pb = ctypes.c_int64()
        _check(lib().ccsd_server_stats(self.s, ctypes.byref(q), ctypes.byref(a), ctypes.byref(pb), ctypes.byref(pa)))
        return {"queued": q.value, "active": a.value, "peak_bytes": pb.value, "peak_active": pa.value}

    def close(self):
        if self.s:
            _check(lib().ccsd_server_destroy(self.s))
            self.s = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
