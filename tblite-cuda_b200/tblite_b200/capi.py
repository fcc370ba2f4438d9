"""ctypes binding of the tblite-b200 C ABI (include/tblite_b200.h).

This is the Python mirror of the reference's singlepoint interface: a
``Calculator`` (xtb_calculator, reference src/xtb.h:105-126) and
``singlepoint_batch`` (xtb_singlepoint, src/xtb.cu:188-434, batched).  All
computation happens in ``lib/libtblite_b200.so`` on the GPU; there is no CPU
fallback -- if the library is missing this module raises on first use.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

PKG = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB_PATH = os.path.join(PKG, "lib", "libtblite_b200.so")
# the checked build (index guards that skip and record out-of-slice accesses)
LIB_CHECK_PATH = os.path.join(PKG, "lib", "libtblite_b200_check.so")
DEFAULT_PARAMS = os.path.join(PKG, "params", "synthetic_hco.tbp")

TB_OK, TB_BAD_INPUT, TB_NOT_SPD, TB_SCF_NOT_CONVERGED = 0, 1, 2, 3
TB_FERMI_NOT_CONVERGED, TB_EIGEN_FAILED, TB_CAPACITY_EXCEEDED = 4, 5, 6
TB_CUDA_ERROR, TB_PARAM_ERROR = 7, 8
STATUS_NAMES = {0: "TB_OK", 1: "TB_BAD_INPUT", 2: "TB_NOT_SPD", 3: "TB_SCF_NOT_CONVERGED",
                4: "TB_FERMI_NOT_CONVERGED", 5: "TB_EIGEN_FAILED", 6: "TB_CAPACITY_EXCEEDED",
                7: "TB_CUDA_ERROR", 8: "TB_PARAM_ERROR"}

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int32)


class Structure(C.Structure):
    _fields_ = [("nat", C.c_int32), ("uhf", C.c_int32), ("charge", C.c_double),
                ("id", _ip), ("xyz", _dp)]


class Options(C.Structure):
    _fields_ = [("accuracy", C.c_double), ("kt", C.c_double), ("max_iter", C.c_int32),
                ("mixer_damping", C.c_double), ("verbosity", C.c_int32), ("use_graphs", C.c_int32),
                ("solver", C.c_int32), ("profile", C.c_int32),
                ("precision", C.c_int32)]


class Result(C.Structure):
    _fields_ = [("energy", C.c_double), ("e_rep", C.c_double), ("e_elec", C.c_double),
                ("e_band", C.c_double), ("e_ts", C.c_double), ("e_es2", C.c_double),
                ("e_aes2", C.c_double), ("e_es3", C.c_double), ("dipole", C.c_double * 3),
                ("scf_error", C.c_double), ("iterations", C.c_int32), ("status", C.c_int32),
                ("nsh", C.c_int32), ("nao", C.c_int32), ("qat", _dp), ("qsh", _dp), ("dpat", _dp),
                ("qpat", _dp), ("gradient", _dp), ("sigma", C.c_double * 9), ("e_disp", C.c_double)]


class Wavefunction(C.Structure):
    """tb_wavefunction: wavefunction_type (reference src/wavefunction/type.h:81-99)."""
    _fields_ = [("guess", C.c_int32), ("nspin", C.c_int32), ("nat", C.c_int32), ("nsh", C.c_int32),
                ("nao", C.c_int32), ("homo", C.c_int32 * 2), ("kt", C.c_double), ("nocc", C.c_double),
                ("nuhf", C.c_double), ("nel", C.c_double * 2), ("n0at", _dp), ("n0sh", _dp), ("emo", _dp),
                ("focc", _dp), ("density", _dp), ("coeff", _dp), ("qat", _dp), ("qsh", _dp), ("dpat", _dp),
                ("qpat", _dp)]


EXPORTS = [
    "tb_calculator_create", "tb_calculator_destroy", "tb_calculator_nspecies", "tb_default_options",
    "tb_last_error", "tb_basis_size", "tb_singlepoint_batch", "tb_batch_create", "tb_batch_run",
    "tb_batch_results", "tb_batch_launches", "tb_batch_destroy", "tb_get_cutoff", "tb_adjacency_list",
    "tb_atomic_properties", "tb_repulsion", "tb_get_hamiltonian", "tb_coulomb_potential",
    "tb_add_pot_to_h1", "tb_sygvd_batch", "tb_fermi_filling", "tb_batch_profile",
    "tb_server_create", "tb_server_submit", "tb_server_step", "tb_server_poll", "tb_server_destroy",
    "tb_batch_set_guess", "tb_batch_wavefunction", "tb_batch_gradient", "tb_sygvd_noalloc",
    "tb_calculator_set_small_solver", "tb_calculator_set_smem_tridiag", "tb_calculator_tuning",
    "tb_bounds_check_build", "tb_bounds_violations", "tb_server_compactions", "tb_dispersion",
    "tb_read_xyz", "tb_calculator_species", "tb_calculator_set_gemm_tiles",
]

_lib = None


class TBError(RuntimeError):
    def __init__(self, status, msg):
        super().__init__(f"{STATUS_NAMES.get(status, status)}: {msg}")
        self.status = status


def load_library(path: str = LIB_PATH):
    """Load libtblite_b200.so (raises if it is missing: there is no fallback)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise RuntimeError(f"tblite-b200 CUDA library not built: {path} (run __graft_entry__.build())")
    L = C.CDLL(path)
    L.tb_last_error.restype = C.c_char_p
    L.tb_get_cutoff.restype = C.c_double
    L.tb_get_cutoff.argtypes = [C.c_void_p, C.c_double]
    L.tb_calculator_create.argtypes = [C.c_char_p, C.POINTER(C.c_void_p)]
    L.tb_calculator_destroy.argtypes = [C.c_void_p]
    L.tb_calculator_nspecies.argtypes = [C.c_void_p]
    L.tb_default_options.argtypes = [C.POINTER(Options)]
    L.tb_batch_launches.restype = C.c_int64
    L.tb_batch_launches.argtypes = [C.c_void_p]
    L.tb_batch_destroy.argtypes = [C.c_void_p]
    L.tb_server_create.argtypes = [C.c_void_p, C.POINTER(Options), C.c_int64, C.c_int32, C.POINTER(C.c_void_p)]
    L.tb_server_submit.argtypes = [C.c_void_p, C.POINTER(Structure), C.POINTER(C.c_int64)]
    L.tb_server_step.argtypes = [C.c_void_p, C.POINTER(C.c_int32), C.POINTER(C.c_int32), C.POINTER(C.c_int64)]
    L.tb_server_poll.argtypes = [C.c_void_p, C.c_int32, C.POINTER(C.c_int64), C.c_void_p]
    L.tb_server_poll.restype = C.c_int32
    L.tb_server_destroy.argtypes = [C.c_void_p]
    L.tb_server_compactions.argtypes = [C.c_void_p]
    L.tb_server_compactions.restype = C.c_int64
    L.tb_calculator_set_small_solver.argtypes = [C.c_void_p, C.c_int32]
    L.tb_calculator_set_smem_tridiag.argtypes = [C.c_void_p, C.c_int32]
    L.tb_calculator_set_gemm_tiles.argtypes = [C.c_void_p, C.c_int32]
    L.tb_bounds_check_build.restype = C.c_int32
    L.tb_calculator_tuning.argtypes = [C.c_void_p, C.c_char_p, C.c_int32]
    L.tb_calculator_tuning.restype = C.c_int32
    _lib = L
    return L


def bounds_violations(reset=True):
    """(count, site, index, lo, hi) of the checked build's index guards (tb_bounds_violations)."""
    v = [C.c_int64(), C.c_int32(), C.c_int64(), C.c_int64(), C.c_int64()]
    check(load_library().tb_bounds_violations(*[C.byref(x) for x in v], C.c_int32(int(reset))), "tb_bounds_violations")
    return tuple(x.value for x in v)


def last_error() -> str:
    return load_library().tb_last_error().decode()


def check(st: int, what: str = ""):
    if st != TB_OK:
        raise TBError(st, f"{what}: {last_error()}")


def default_options(**kw) -> Options:
    o = Options()
    load_library().tb_default_options(C.byref(o))
    for k, v in kw.items():
        setattr(o, k, v)
    return o


def _record_dtype(cls, kinds):
    """numpy view of a ctypes record array: same offsets and itemsize; pointer
    fields as unsigned integers (addresses)."""
    names = [f[0] for f in cls._fields_]
    return np.dtype({"names": names, "formats": [kinds[k] for k in names],
                     "offsets": [getattr(cls, k).offset for k in names], "itemsize": C.sizeof(cls)})


_STRUCT_DT = _record_dtype(Structure, {"nat": np.int32, "uhf": np.int32, "charge": np.float64,
                                       "id": np.uintp, "xyz": np.uintp})
_RESULT_DT = _record_dtype(Result, dict(
    {k: np.float64 for k in ("energy", "e_rep", "e_elec", "e_band", "e_ts", "e_es2", "e_aes2", "e_es3",
                             "scf_error", "e_disp")},
    dipole=(np.float64, 3), iterations=np.int32, status=np.int32, nsh=np.int32, nao=np.int32,
    qat=np.uintp, qsh=np.uintp, dpat=np.uintp, qpat=np.uintp, gradient=np.uintp, sigma=(np.float64, 9)))


def _structs(mols):
    """Pack Molecule-like objects (id, xyz, charge, uhf) into tb_structure records.
    All species ids and coordinates go into two contiguous arrays; the records
    are filled through a numpy view of the ctypes array (pointer = base address
    + offset), so the cost does not grow with a Python loop of ctypes calls."""
    n = len(mols)
    arr = (Structure * n)()
    if n == 0:
        return arr, ()
    idl = [m.id for m in mols]
    xyl = [m.xyz for m in mols]
    if all(isinstance(a, np.ndarray) and a.ndim == 1 for a in idl) and \
            all(isinstance(x, np.ndarray) and x.ndim == 2 and x.shape[1] == 3 for x in xyl):
        # arrays already shaped as Molecule holds them: one concatenation each
        ids = np.ascontiguousarray(np.concatenate(idl), dtype=np.int32)
        xyz = np.ascontiguousarray(np.concatenate(xyl), dtype=np.float64)
    else:
        idl = [np.asarray(a, np.int32).ravel() for a in idl]
        ids = np.ascontiguousarray(np.concatenate(idl))
        xyz = np.ascontiguousarray(np.concatenate([np.asarray(x, np.float64).reshape(-1, 3) for x in xyl]))
    nat = np.fromiter((len(a) for a in idl), np.int64, n)
    off = np.zeros(n, np.int64)
    np.cumsum(nat[:-1], out=off[1:])
    v = np.frombuffer(arr, dtype=_STRUCT_DT)
    v["nat"] = nat
    v["uhf"] = [int(getattr(m, "uhf", 0)) for m in mols]
    v["charge"] = [float(getattr(m, "charge", 0.0)) for m in mols]
    v["id"] = ids.ctypes.data + ids.itemsize * off
    v["xyz"] = xyz.ctypes.data + 3 * xyz.itemsize * off
    return arr, (ids, xyz, nat, off)


class Calculator:
    """GFN2-shaped xTB calculator bound to one parameter file (tb_calculator)."""

    def __init__(self, param_file: str = DEFAULT_PARAMS):
        L = load_library()
        h = C.c_void_p()
        check(L.tb_calculator_create(param_file.encode(), C.byref(h)), "tb_calculator_create")
        self.h = h

    def __del__(self):
        try:
            if getattr(self, "h", None) and self.h.value:
                load_library().tb_calculator_destroy(self.h)
                self.h = None
        except Exception:
            pass

    def basis_size(self, mol):
        arr, keep = _structs([mol])
        nsh, nao = C.c_int32(), C.c_int32()
        check(load_library().tb_basis_size(self.h, C.byref(arr[0]), C.byref(nsh), C.byref(nao)),
              "tb_basis_size")
        return nsh.value, nao.value

    def _species_basis(self):
        """Shells and AOs per species (from one-atom structures, once)."""
        if getattr(self, "_sp_basis", None) is None:
            ns = load_library().tb_calculator_nspecies(self.h)
            self._sp_basis = np.array([self.basis_size(_Atom(z)) for z in range(ns)], np.int64).reshape(-1, 2)
        return self._sp_basis

    def set_small_solver(self, jacobi_max: int):
        """Eigensolver variant of small structures: -1 measured choice (default),
        0 never the one-warp Jacobi solver, 1..32 Jacobi up to that many AOs."""
        check(load_library().tb_calculator_set_small_solver(self.h, C.c_int32(jacobi_max)),
              "tb_calculator_set_small_solver")

    def set_gemm_tiles(self, max_n32: int):
        """FP64 GEMM tile shape per structure: -1 the measured choice
        (default), 0 always 64 x 64, N > 0 32 x 32 tiles up to N AOs.  Both
        shapes give the same bits."""
        check(load_library().tb_calculator_set_gemm_tiles(self.h, C.c_int32(max_n32)),
              "tb_calculator_set_gemm_tiles")

    def set_smem_tridiag(self, min_n):
        """FP64 tridiagonalisation in cluster shared memory (k_trid_smem) for
        structures of at least min_n AOs (and 64..560): lower latency per
        structure, more SM time.  True means every size from 64, False or 0
        none (the default)."""
        if min_n is True:
            min_n = 64
        check(load_library().tb_calculator_set_smem_tridiag(self.h, C.c_int32(int(min_n))),
              "tb_calculator_set_smem_tridiag")

    def molecule_from_xyz(self, path: str, charge: float = 0.0, uhf: int = 0):
        """A structure from an XYZ file, species mapped by this calculator's parameter file."""
        from .geometry import Molecule
        z, xyz, comment = read_xyz(path)
        L = load_library()
        L.tb_calculator_species.argtypes = [C.c_void_p, C.c_int32]
        sp = np.array([L.tb_calculator_species(self.h, C.c_int32(int(x))) for x in z], np.int32)
        if (sp < 0).any():
            raise TBError(TB_BAD_INPUT, f"{path}: element Z={int(z[sp < 0][0])} is not in the parameter file")
        return Molecule(sp, xyz, charge=charge, uhf=uhf, label=comment.strip() or os.path.basename(path))

    def tuning(self) -> dict:
        """The autotuner's measurements and choices (tb_calculator_tuning)."""
        import json
        L = load_library()
        n = L.tb_calculator_tuning(self.h, None, C.c_int32(0))
        buf = C.create_string_buffer(n + 1)
        L.tb_calculator_tuning(self.h, buf, C.c_int32(n + 1))
        return json.loads(buf.value.decode())

    def cutoff(self, accuracy=1.0):
        return load_library().tb_get_cutoff(self.h, C.c_double(accuracy))

    def singlepoint_batch(self, mols, stream=None, raise_on_error=False, wavefunction=False, guess=None, nspin=1,
                          gradient=False, **opts):
        """Run xtb_singlepoint for every structure; returns a list of result dicts.

        wavefunction=True adds r["wfn"] (the tb_wavefunction record as a dict:
        emo, focc, density, coeff, n0at, n0sh, nel, homo, ...).  guess is None or
        a list (one entry per structure, None for the default start) of dicts
        with qsh, dpat and qpat to start the SCF from, e.g. an earlier result.
        nspin=2 returns the wavefunction in the open-shell representation
        (leading channel index on every array, see tb_wavefunction).
        gradient=True adds r["gradient"] ([nat][3], Eh/Bohr) and r["sigma"] (3x3)."""
        L = load_library()
        arr, keep = _structs(mols)
        o = default_options(**opts)
        n = len(mols)
        res = (Result * n)()
        # output arrays for all structures at once; each structure gets views
        tab = self._species_basis()
        if n:
            ids, _, nat, off = keep
            if ids.size and (ids.min() < 0 or ids.max() >= len(tab)):
                for m in mols:  # raises the library's own error for the bad species
                    self.basis_size(m)
            owner = np.repeat(np.arange(n), nat)
            nsh = np.bincount(owner, weights=tab[ids, 0], minlength=n).astype(np.int64)
        else:
            nat = off = nsh = np.zeros(0, np.int64)
        soff = np.zeros(n, np.int64)
        if n:
            np.cumsum(nsh[:-1], out=soff[1:])
        na, ns = int(nat.sum()), int(nsh.sum())
        qat, qsh, dpat, qpat = np.zeros(na), np.zeros(ns), np.zeros((na, 3)), np.zeros((na, 6))
        grad = np.zeros((na, 3)) if gradient else None
        v = np.frombuffer(res, dtype=_RESULT_DT) if n else None
        if n:
            v["qat"] = qat.ctypes.data + 8 * off
            v["qsh"] = qsh.ctypes.data + 8 * soff
            v["dpat"] = dpat.ctypes.data + 24 * off
            v["qpat"] = qpat.ctypes.data + 48 * off
            v["gradient"] = grad.ctypes.data + 24 * off if gradient else 0
        wfn, wbufs = None, None
        if n and (wavefunction or guess is not None):
            wfn, wbufs = _wavefunction_records(self, mols, guess, wavefunction, nspin)
        st = L.tb_singlepoint_batch(self.h, arr, C.c_int32(n), C.byref(o), wfn, res, C.c_void_p(stream or 0))
        if st not in (TB_OK,) and (raise_on_error or st in (TB_BAD_INPUT, TB_CUDA_ERROR,
                                                            TB_CAPACITY_EXCEEDED, TB_PARAM_ERROR)):
            check(st, "tb_singlepoint_batch")
        if not n:
            return []
        # each field converted once for all structures (numpy scalar access per field is slow)
        keys = ("energy", "e_rep", "e_elec", "e_band", "e_ts", "e_es2", "e_aes2", "e_es3", "scf_error",
                "e_disp", "iterations", "status", "nsh", "nao")
        # (dicts from zipped columns and the per-structure views by list
        # comprehension: about half the cost of a per-structure loop of dict
        # comprehensions and slices)
        out = [dict(zip(keys, vals)) for vals in zip(*[v[k].tolist() for k in keys])]
        a0s, a1s = off.tolist(), (off + nat).tolist()
        s0s, s1s = soff.tolist(), (soff + nsh).tolist()
        views = {"dipole": list(v["dipole"].copy()),
                 "qat": [qat[a:b] for a, b in zip(a0s, a1s)], "qsh": [qsh[a:b] for a, b in zip(s0s, s1s)],
                 "dpat": [dpat[a:b] for a, b in zip(a0s, a1s)], "qpat": [qpat[a:b] for a, b in zip(a0s, a1s)]}
        if gradient:
            views["gradient"] = [grad[a:b] for a, b in zip(a0s, a1s)]
            views["sigma"] = list(v["sigma"].reshape(n, 3, 3).copy())
        for k, col in views.items():
            for d, x in zip(out, col):
                d[k] = x
        if wavefunction:
            for i, d in enumerate(out):
                w = wfn[i]
                d["wfn"] = dict(wbufs[i], nspin=w.nspin, nat=w.nat, nsh=w.nsh, nao=w.nao, homo=list(w.homo),
                                kt=w.kt, nocc=w.nocc, nuhf=w.nuhf, nel=list(w.nel))
        return out


class _Atom:
    """One atom of species z at the origin (for per-species basis sizes)."""

    def __init__(self, z):
        self.id = np.array([z], np.int32)
        self.xyz = np.zeros((1, 3))
        self.nat = 1


def _result_dict(r, b):
    d = dict(energy=r.energy, e_rep=r.e_rep, e_elec=r.e_elec, e_band=r.e_band, e_ts=r.e_ts,
             e_es2=r.e_es2, e_aes2=r.e_aes2, e_es3=r.e_es3, e_disp=r.e_disp, dipole=np.array(r.dipole[:]),
             scf_error=r.scf_error, iterations=r.iterations, status=r.status, nsh=r.nsh, nao=r.nao)
    d.update(b)
    return d


def _wavefunction_records(calc, mols, guess, outputs, nspin=1):
    """tb_wavefunction records for mols: output arrays when `outputs` (with a
    leading channel index for nspin = 2), the caller's starting moments where
    guess[i] is given."""
    n = len(mols)
    rec = (Wavefunction * n)()
    bufs = []
    ch = (2,) if nspin == 2 else ()
    for i, m in enumerate(mols):
        nsh, nao = calc.basis_size(m)
        b = {}
        rec[i].nspin = nspin
        if outputs:
            b = dict(n0at=np.zeros(m.nat), n0sh=np.zeros(nsh), emo=np.zeros(ch + (nao,)), focc=np.zeros(ch + (nao,)),
                     density=np.zeros(ch + (nao, nao)), coeff=np.zeros(ch + (nao, nao)), qat=np.zeros(ch + (m.nat,)),
                     qsh=np.zeros(ch + (nsh,)), dpat=np.zeros(ch + (m.nat, 3)), qpat=np.zeros(ch + (m.nat, 6)))
        g = guess[i] if guess is not None else None
        if g is not None:
            for k, shape in (("qsh", (nsh,)), ("dpat", (m.nat, 3)), ("qpat", (m.nat, 6))):
                a = np.ascontiguousarray(np.array(g[k], np.float64).reshape(shape))
                if k in b:
                    b[k].reshape((-1,) + shape)[0][...] = a  # channel 0 (total) is the guess
                else:
                    b[k] = a
            rec[i].guess = 1
        for k, a in b.items():
            setattr(rec[i], k, a.ctypes.data_as(_dp))
        bufs.append(b)
    return rec, bufs


class Batch:
    """Device-resident batch (tb_batch): geometry uploaded once, run on device."""

    def __init__(self, calc: Calculator, mols, **opts):
        L = load_library()
        self.calc = calc
        self.mols = mols
        self._arr, self._keep = _structs(mols)
        o = default_options(**opts)
        h = C.c_void_p()
        check(L.tb_batch_create(calc.h, self._arr, C.c_int32(len(mols)), C.byref(o), C.byref(h)),
              "tb_batch_create")
        self.h = h

    def run(self, stream=None):
        st = load_library().tb_batch_run(self.h, C.c_void_p(stream or 0))
        check(st, "tb_batch_run")

    def launches(self) -> int:
        return int(load_library().tb_batch_launches(self.h))

    def profile(self):
        """Per kernel class of the last run: {name: (launches, ms, work, unit)} (needs profile=1)."""
        n = 64
        names = C.create_string_buffer(32 * n)
        la = (C.c_int64 * n)()
        ms = (C.c_double * n)()
        wk = (C.c_double * n)()
        un = (C.c_int32 * n)()
        k = load_library().tb_batch_profile(self.h, C.c_int32(n), names, la, ms, wk, un)
        out = {}
        for i in range(k):
            nm = names.raw[32 * i:32 * (i + 1)].split(b"\0", 1)[0].decode()
            out[nm] = (int(la[i]), float(ms[i]), float(wk[i]), {0: None, 1: "flop", 2: "byte"}[un[i]])
        return out

    def gradient(self, stream=None):
        """Analytic gradient of the last run: ([nat_tot][3] packed over the batch, [nmol][3][3] sigma)."""
        na = sum(m.nat for m in self.mols)
        g = np.zeros((na, 3))
        sg = np.zeros((len(self.mols), 3, 3))
        check(load_library().tb_batch_gradient(self.h, g.ctypes.data_as(_dp), sg.ctypes.data_as(_dp),
                                                C.c_void_p(stream or 0)), "tb_batch_gradient")
        return g, sg

    def results(self, stream=None):
        L = load_library()
        res = (Result * len(self.mols))()
        bufs = []
        for i, m in enumerate(self.mols):
            nsh, nao = self.calc.basis_size(m)
            b = dict(qat=np.zeros(m.nat), qsh=np.zeros(nsh), dpat=np.zeros((m.nat, 3)),
                     qpat=np.zeros((m.nat, 6)))
            bufs.append(b)
            res[i].qat = b["qat"].ctypes.data_as(_dp)
            res[i].qsh = b["qsh"].ctypes.data_as(_dp)
            res[i].dpat = b["dpat"].ctypes.data_as(_dp)
            res[i].qpat = b["qpat"].ctypes.data_as(_dp)
        L.tb_batch_results(self.h, res, C.c_void_p(stream or 0))
        return [_result_dict(r, b) for r, b in zip(res, bufs)]

    def __del__(self):
        try:
            if getattr(self, "h", None) and self.h.value:
                load_library().tb_batch_destroy(self.h)
                self.h = None
        except Exception:
            pass


class Server:
    """Continuous-batching request loop (tb_server): submit() queues a
    structure, step() admits queued requests within the device-memory budget
    and runs one SCF iteration of every resident micro-batch, poll() returns
    finished results as (ticket, result dict)."""

    def __init__(self, calc: Calculator, hbm_budget_bytes: int, max_batch: int = 256, **opts):
        L = load_library()
        self.calc = calc
        o = default_options(**opts)
        h = C.c_void_p()
        check(L.tb_server_create(calc.h, C.byref(o), C.c_int64(int(hbm_budget_bytes)), C.c_int32(max_batch),
                                 C.byref(h)), "tb_server_create")
        self.h = h
        self._sizes = {}

    def submit(self, mol) -> int:
        arr, keep = _structs([mol])
        t = C.c_int64()
        check(load_library().tb_server_submit(self.h, C.byref(arr[0]), C.byref(t)), "tb_server_submit")
        self._sizes[t.value] = (mol.nat, self.calc.basis_size(mol)[0])
        return t.value

    def step(self):
        """Returns (requests resident on the device, requests queued, workspace bytes resident)."""
        nr, nq, nb = C.c_int32(), C.c_int32(), C.c_int64()
        check(load_library().tb_server_step(self.h, C.byref(nr), C.byref(nq), C.byref(nb)), "tb_server_step")
        return nr.value, nq.value, nb.value

    def compactions(self) -> int:
        """Micro-batches moved to their unfinished structures so far (tb_server_compactions)."""
        return int(load_library().tb_server_compactions(self.h))

    def poll(self, max_results: int = 4096):
        L = load_library()
        out = []
        while True:
            # one result at a time so that every array buffer has its structure's size
            t = C.c_int64()
            res = (Result * 1)()
            pending = [k for k in self._sizes]
            if not pending:
                break
            # sizes are per ticket: peek by polling into the largest buffers needed, then trim
            nat = max(v[0] for v in self._sizes.values())
            nsh = max(v[1] for v in self._sizes.values())
            b = dict(qat=np.zeros(nat), qsh=np.zeros(nsh), dpat=np.zeros((nat, 3)), qpat=np.zeros((nat, 6)))
            res[0].qat = b["qat"].ctypes.data_as(_dp)
            res[0].qsh = b["qsh"].ctypes.data_as(_dp)
            res[0].dpat = b["dpat"].ctypes.data_as(_dp)
            res[0].qpat = b["qpat"].ctypes.data_as(_dp)
            k = L.tb_server_poll(self.h, 1, C.byref(t), res)
            if k == 0 or len(out) >= max_results:
                break
            na, ns = self._sizes.pop(t.value)
            b = dict(qat=b["qat"][:na].copy(), qsh=b["qsh"][:ns].copy(), dpat=b["dpat"][:na].copy(),
                     qpat=b["qpat"][:na].copy())
            out.append((t.value, _result_dict(res[0], b)))
        return out

    def __del__(self):
        try:
            if getattr(self, "h", None) and self.h.value:
                load_library().tb_server_destroy(self.h)
                self.h = None
        except Exception:
            pass


# ---------------------------------------------------------------- stage calls
def _one(mol):
    arr, keep = _structs([mol])
    return arr, keep


def adjacency_list(calc: Calculator, mol, cutoff: float):
    arr, keep = _one(mol)
    nat = mol.nat
    cap = max(1, nat * (nat - 1) // 2)
    inl, nnl = np.zeros(nat, np.int32), np.zeros(nat, np.int32)
    nlat = np.zeros(cap, np.int32)
    npair = C.c_int32()
    check(load_library().tb_adjacency_list(calc.h, C.byref(arr[0]), C.c_double(cutoff), inl.ctypes.data_as(_ip),
                                           nnl.ctypes.data_as(_ip), nlat.ctypes.data_as(_ip), C.c_int32(cap),
                                           C.byref(npair)), "tb_adjacency_list")
    return inl, nnl, nlat[:npair.value].copy()


def atomic_properties(calc: Calculator, mol):
    arr, keep = _one(mol)
    nsh, _ = calc.basis_size(mol)
    cn, mrad, se = np.zeros(mol.nat), np.zeros(mol.nat), np.zeros(nsh)
    check(load_library().tb_atomic_properties(calc.h, C.byref(arr[0]), cn.ctypes.data_as(_dp),
                                              mrad.ctypes.data_as(_dp), se.ctypes.data_as(_dp)),
          "tb_atomic_properties")
    return cn, mrad, se


def repulsion(calc: Calculator, mol):
    arr, keep = _one(mol)
    e = np.zeros(mol.nat)
    check(load_library().tb_repulsion(calc.h, C.byref(arr[0]), e.ctypes.data_as(_dp)), "tb_repulsion")
    return e


def read_xyz(path: str):
    """An XYZ file through tb_read_xyz: (atomic numbers, coordinates [nat][3] in Bohr, comment line)."""
    L = load_library()
    L.tb_read_xyz.argtypes = [C.c_char_p, C.c_int32, C.POINTER(C.c_int32), C.c_void_p, C.c_void_p, C.c_char_p,
                              C.c_int32]
    nat = C.c_int32()
    st = L.tb_read_xyz(path.encode(), 0, C.byref(nat), None, None, None, 0)
    if st not in (TB_OK, TB_CAPACITY_EXCEEDED):
        check(st, "tb_read_xyz")
    z, xyz = np.zeros(nat.value, np.int32), np.zeros((nat.value, 3))
    comment = C.create_string_buffer(4096)
    check(L.tb_read_xyz(path.encode(), nat.value, C.byref(nat), z.ctypes.data_as(C.c_void_p),
                        xyz.ctypes.data_as(C.c_void_p), comment, 4096), "tb_read_xyz")
    return z, xyz, comment.value.decode(errors="replace")


def dispersion(calc: Calculator, mol):
    """D4 dispersion (tb_dispersion): per-atom energies, gradient [nat][3], virial [3][3]."""
    arr, keep = _one(mol)
    e, g, s = np.zeros(mol.nat), np.zeros((mol.nat, 3)), np.zeros((3, 3))
    check(load_library().tb_dispersion(calc.h, C.byref(arr[0]), e.ctypes.data_as(_dp), g.ctypes.data_as(_dp),
                                       s.ctypes.data_as(_dp)), "tb_dispersion")
    return e, g, s


def get_hamiltonian(calc: Calculator, mol):
    arr, keep = _one(mol)
    _, n = calc.basis_size(mol)
    S, H0, D, Q = np.zeros((n, n)), np.zeros((n, n)), np.zeros((3, n, n)), np.zeros((6, n, n))
    check(load_library().tb_get_hamiltonian(calc.h, C.byref(arr[0]), *[a.ctypes.data_as(_dp) for a in (S, H0, D, Q)]),
          "tb_get_hamiltonian")
    return S, H0, D, Q


def coulomb_potential(calc: Calculator, mol, qsh, dpat, qpat):
    arr, keep = _one(mol)
    nsh, _ = calc.basis_size(mol)
    qsh, dpat, qpat = (np.ascontiguousarray(a, np.float64) for a in (qsh, dpat, qpat))
    vsh, vat, vdp, vqp = np.zeros(nsh), np.zeros(mol.nat), np.zeros((mol.nat, 3)), np.zeros((mol.nat, 6))
    check(load_library().tb_coulomb_potential(calc.h, C.byref(arr[0]),
                                              *[a.ctypes.data_as(_dp) for a in (qsh, dpat, qpat, vsh, vat, vdp, vqp)]),
          "tb_coulomb_potential")
    return vsh, vat, vdp, vqp


def add_pot_to_h1(calc: Calculator, mol, S, H0, D, Q, vsh, vat, vdp, vqp):
    arr, keep = _one(mol)
    ins = [np.ascontiguousarray(a, np.float64) for a in (S, H0, D, Q, vsh, vat, vdp, vqp)]
    F = np.zeros_like(ins[0])
    check(load_library().tb_add_pot_to_h1(calc.h, C.byref(arr[0]), *[a.ctypes.data_as(_dp) for a in ins],
                                          F.ctypes.data_as(_dp)), "tb_add_pot_to_h1")
    return F


def sygvd_batch(Hs, Ss):
    """Generalized eigenproblems H C = S C e for a list of (n_i x n_i) pairs."""
    n = np.array([h.shape[0] for h in Hs], np.int32)
    H = np.ascontiguousarray(np.concatenate([np.ravel(h) for h in Hs]), np.float64)
    S = np.ascontiguousarray(np.concatenate([np.ravel(s) for s in Ss]), np.float64)
    w = np.zeros(int(n.sum()))
    Cm = np.zeros_like(H)
    st = load_library().tb_sygvd_batch(C.c_int32(len(n)), n.ctypes.data_as(_ip), H.ctypes.data_as(_dp),
                                       S.ctypes.data_as(_dp), w.ctypes.data_as(_dp), Cm.ctypes.data_as(_dp))
    out, wo, co = [], 0, 0
    for k in n:
        out.append((w[wo:wo + k].copy(), Cm[co:co + k * k].reshape(k, k).copy()))
        wo += k
        co += k * k
    return st, out


def fermi_filling(nel, kt, emo):
    emo = np.ascontiguousarray(emo, np.float64)
    occ = np.zeros_like(emo)
    ef, ts = C.c_double(), C.c_double()
    st = load_library().tb_fermi_filling(C.c_int32(len(emo)), C.c_double(nel), C.c_double(kt),
                                         emo.ctypes.data_as(_dp), occ.ctypes.data_as(_dp), C.byref(ef),
                                         C.byref(ts))
    return st, occ, ef.value, ts.value

