"""ctypes wrapper of the FP64 CPU oracle (liboracle.so) -- TEST INFRASTRUCTURE ONLY.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg import
this module; the CUDA product library never does.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "liboracle.so")

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int)


class Options(C.Structure):
    _fields_ = [("accuracy", C.c_double), ("kt", C.c_double), ("max_iter", C.c_int),
                ("damping", C.c_double), ("verbosity", C.c_int)]


class Result(C.Structure):
    _fields_ = [("energy", C.c_double), ("e_rep", C.c_double), ("e_elec", C.c_double),
                ("e_band", C.c_double), ("e_ts", C.c_double), ("e_es2", C.c_double),
                ("e_aes2", C.c_double), ("e_es3", C.c_double), ("dipole", C.c_double * 3),
                ("iterations", C.c_int), ("status", C.c_int), ("nsh", C.c_int), ("nao", C.c_int),
                ("e_disp", C.c_double)]


def _d(a):
    return a.ctypes.data_as(_dp)


def _i(a):
    return a.ctypes.data_as(_ip)


_lib = None


def use_library(path: str):
    """Load the oracle from another build of the same source (e.g. the
    -march=native one the CPU baseline times); call before the first use."""
    global LIB
    if _lib is not None:
        raise RuntimeError("oracle library already loaded")
    LIB = path


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB):
            raise RuntimeError(f"oracle library missing: {LIB} (run make -C oracle)")
        L = C.CDLL(LIB)
        L.orc_params_load.restype = C.c_void_p
        L.orc_params_load.argtypes = [C.c_char_p, C.c_char_p, C.c_int]
        L.orc_params_free.argtypes = [C.c_void_p]
        L.orc_cutoff.restype = C.c_double
        L.orc_cutoff.argtypes = [C.c_void_p, C.c_double]
        for name in ("orc_basis_size", "orc_basis_maps", "orc_coordination_number", "orc_mrad",
                     "orc_selfenergy", "orc_hamiltonian", "orc_repulsion", "orc_coulomb_matrices",
                     "orc_coulomb_potential", "orc_coulomb_energy", "orc_fock", "orc_mulliken",
                     "orc_singlepoint", "orc_singlepoint_batch", "orc_singlepoint_spin", "orc_singlepoint_gradient", "orc_multipole_cgto", "orc_nspecies",
                     "orc_dispersion", "orc_has_dispersion"):
            getattr(L, name).argtypes = None
            getattr(L, name).restype = C.c_int
        L.orc_default_options.argtypes = [C.POINTER(Options)]
        _lib = L
    return _lib


def default_options(**kw) -> Options:
    o = Options()
    lib().orc_default_options(C.byref(o))
    for k, v in kw.items():
        setattr(o, k, v)
    return o


class Oracle:
    """FP64 reference calculator bound to one parameter file."""

    def __init__(self, param_file: str):
        err = C.create_string_buffer(512)
        h = lib().orc_params_load(param_file.encode(), err, 512)
        if not h:
            raise RuntimeError(err.value.decode())
        self.h = C.c_void_p(h)

    def __del__(self):
        try:
            if getattr(self, "h", None):
                lib().orc_params_free(self.h)
        except Exception:
            pass

    # --- basis
    def basis_size(self, ids):
        ids = np.ascontiguousarray(ids, np.int32)
        nsh, nao = C.c_int(), C.c_int()
        st = lib().orc_basis_size(self.h, C.c_int(len(ids)), _i(ids), C.byref(nsh), C.byref(nao))
        if st:
            raise ValueError("bad species")
        return nsh.value, nao.value

    def basis_maps(self, ids):
        ids = np.ascontiguousarray(ids, np.int32)
        nsh, nao = self.basis_size(ids)
        nat = len(ids)
        out = dict(ish_at=np.zeros(nat, np.int32), iao_sh=np.zeros(nsh, np.int32),
                   ao2at=np.zeros(nao, np.int32), ao2sh=np.zeros(nao, np.int32),
                   sh2at=np.zeros(nsh, np.int32), ang_sh=np.zeros(nsh, np.int32))
        lib().orc_basis_maps(self.h, C.c_int(nat), _i(ids), *[_i(out[k]) for k in
                             ("ish_at", "iao_sh", "ao2at", "ao2sh", "sh2at", "ang_sh")])
        return out

    def cutoff(self, accuracy=1.0):
        return lib().orc_cutoff(self.h, C.c_double(accuracy))

    # --- stages
    @staticmethod
    def adjacency_list(xyz, cutoff):
        xyz = np.ascontiguousarray(xyz, np.float64)
        nat = xyz.shape[0]
        cap = nat * (nat + 1) // 2
        inl, nnl = np.zeros(nat, np.int32), np.zeros(nat, np.int32)
        nlat, nltr = np.zeros(max(cap, 1), np.int32), np.zeros(max(cap, 1), np.int32)
        npair = C.c_int()
        lib().orc_adjacency_list(C.c_int(nat), _d(xyz), C.c_double(cutoff), _i(inl), _i(nnl), _i(nlat),
                                 _i(nltr), C.c_int(cap), C.byref(npair))
        return inl, nnl, nlat[:npair.value].copy(), nltr[:npair.value].copy()

    def coordination_number(self, ids, xyz):
        ids = np.ascontiguousarray(ids, np.int32); xyz = np.ascontiguousarray(xyz, np.float64)
        cn = np.zeros(len(ids))
        lib().orc_coordination_number(self.h, C.c_int(len(ids)), _i(ids), _d(xyz), _d(cn))
        return cn

    def mrad(self, ids, cn):
        ids = np.ascontiguousarray(ids, np.int32); cn = np.ascontiguousarray(cn, np.float64)
        out = np.zeros(len(ids))
        lib().orc_mrad(self.h, C.c_int(len(ids)), _i(ids), _d(cn), _d(out))
        return out

    def selfenergy(self, ids, cn):
        ids = np.ascontiguousarray(ids, np.int32); cn = np.ascontiguousarray(cn, np.float64)
        nsh, _ = self.basis_size(ids)
        out = np.zeros(nsh)
        lib().orc_selfenergy(self.h, C.c_int(len(ids)), _i(ids), _d(cn), _d(out))
        return out

    def hamiltonian(self, ids, xyz):
        ids = np.ascontiguousarray(ids, np.int32); xyz = np.ascontiguousarray(xyz, np.float64)
        _, n = self.basis_size(ids)
        S, H0 = np.zeros((n, n)), np.zeros((n, n))
        D, Q = np.zeros((3, n, n)), np.zeros((6, n, n))
        lib().orc_hamiltonian(self.h, C.c_int(len(ids)), _i(ids), _d(xyz), _d(S), _d(H0), _d(D), _d(Q))
        return S, H0, D, Q

    def repulsion(self, ids, xyz):
        ids = np.ascontiguousarray(ids, np.int32); xyz = np.ascontiguousarray(xyz, np.float64)
        e = np.zeros(len(ids))
        lib().orc_repulsion(self.h, C.c_int(len(ids)), _i(ids), _d(xyz), _d(e))
        return e

    def dispersion(self, ids, xyz):
        """D4 dispersion (orc_dispersion): per-atom energies, gradient [nat][3], virial [3][3]."""
        ids = np.ascontiguousarray(ids, np.int32); xyz = np.ascontiguousarray(xyz, np.float64)
        e, g, s = np.zeros(len(ids)), np.zeros((len(ids), 3)), np.zeros((3, 3))
        lib().orc_dispersion(self.h, C.c_int(len(ids)), _i(ids), _d(xyz), _d(e), _d(g), _d(s))
        return e, g, s

    def has_dispersion(self):
        return bool(lib().orc_has_dispersion(self.h))

    def coulomb_matrices(self, ids, xyz):
        ids = np.ascontiguousarray(ids, np.int32); xyz = np.ascontiguousarray(xyz, np.float64)
        nsh, _ = self.basis_size(ids)
        nat = len(ids)
        g = np.zeros((nsh, nsh)); sd = np.zeros((nat, nat, 3)); dd = np.zeros((nat, 3, nat, 3))
        sq = np.zeros((nat, nat, 6))
        lib().orc_coulomb_matrices(self.h, C.c_int(nat), _i(ids), _d(xyz), _d(g), _d(sd), _d(dd), _d(sq))
        return g, sd, dd, sq

    def coulomb_potential(self, ids, xyz, qsh, dpat, qpat):
        ids = np.ascontiguousarray(ids, np.int32); xyz = np.ascontiguousarray(xyz, np.float64)
        nat = len(ids); nsh, _ = self.basis_size(ids)
        qsh, dpat, qpat = (np.ascontiguousarray(a, np.float64) for a in (qsh, dpat, qpat))
        vsh, vat, vdp, vqp = np.zeros(nsh), np.zeros(nat), np.zeros((nat, 3)), np.zeros((nat, 6))
        lib().orc_coulomb_potential(self.h, C.c_int(nat), _i(ids), _d(xyz), _d(qsh), _d(dpat), _d(qpat),
                                    _d(vsh), _d(vat), _d(vdp), _d(vqp))
        return vsh, vat, vdp, vqp

    def coulomb_energy(self, ids, xyz, qsh, dpat, qpat):
        ids = np.ascontiguousarray(ids, np.int32); xyz = np.ascontiguousarray(xyz, np.float64)
        qsh, dpat, qpat = (np.ascontiguousarray(a, np.float64) for a in (qsh, dpat, qpat))
        e = [C.c_double() for _ in range(3)]
        lib().orc_coulomb_energy(self.h, C.c_int(len(ids)), _i(ids), _d(xyz), _d(qsh), _d(dpat), _d(qpat),
                                 *[C.byref(x) for x in e])
        return tuple(x.value for x in e)

    def fock(self, ids, S, H0, D, Q, vsh, vat, vdp, vqp):
        ids = np.ascontiguousarray(ids, np.int32)
        arrs = [np.ascontiguousarray(a, np.float64) for a in (S, H0, D, Q, vsh, vat, vdp, vqp)]
        F = np.zeros_like(arrs[0])
        lib().orc_fock(self.h, C.c_int(len(ids)), _i(ids), *[_d(a) for a in arrs], _d(F))
        return F

    @staticmethod
    def sygvd(H, S):
        H = np.ascontiguousarray(H, np.float64); S = np.ascontiguousarray(S, np.float64)
        n = H.shape[0]
        w, Cm = np.zeros(n), np.zeros((n, n))
        st = lib().orc_sygvd(C.c_int(n), _d(H), _d(S), _d(w), _d(Cm))
        return st, w, Cm

    @staticmethod
    def fermi(nel, kt, emo):
        emo = np.ascontiguousarray(emo, np.float64)
        occ = np.zeros_like(emo)
        ef, ts = C.c_double(), C.c_double()
        st = lib().orc_fermi(C.c_int(len(emo)), C.c_double(nel), C.c_double(kt), _d(emo), _d(occ),
                             C.byref(ef), C.byref(ts))
        return st, occ, ef.value, ts.value

    def mulliken(self, ids, S, D, Q, P):
        ids = np.ascontiguousarray(ids, np.int32)
        nat = len(ids); nsh, _ = self.basis_size(ids)
        arrs = [np.ascontiguousarray(a, np.float64) for a in (S, D, Q, P)]
        qsh, qat, dpat, qpat = np.zeros(nsh), np.zeros(nat), np.zeros((nat, 3)), np.zeros((nat, 6))
        lib().orc_mulliken(self.h, C.c_int(nat), _i(ids), *[_d(a) for a in arrs], _d(qsh), _d(qat),
                           _d(dpat), _d(qpat))
        return qsh, qat, dpat, qpat

    def multipole_cgto(self, jsp, jsh, isp, ish, r2, vec, intcut=25.0):
        vec = np.ascontiguousarray(vec, np.float64)
        s, d, q = np.zeros(25), np.zeros(75), np.zeros(150)
        lib().orc_multipole_cgto(self.h, C.c_int(jsp), C.c_int(jsh), C.c_int(isp), C.c_int(ish),
                                 C.c_double(r2), _d(vec), C.c_double(intcut), _d(s), _d(d), _d(q))
        return s, d, q

    # --- singlepoint
    def singlepoint(self, mol, **opts):
        ids = np.ascontiguousarray(mol.id, np.int32); xyz = np.ascontiguousarray(mol.xyz, np.float64)
        nat = len(ids); nsh, nao = self.basis_size(ids)
        o = default_options(**opts)
        r = Result()
        out = dict(qat=np.zeros(nat), qsh=np.zeros(nsh), dpat=np.zeros((nat, 3)), qpat=np.zeros((nat, 6)),
                   emo=np.zeros(nao), P=np.zeros((nao, nao)))
        lib().orc_singlepoint(self.h, C.c_int(nat), _i(ids), _d(xyz), C.c_double(mol.charge),
                              C.c_int(mol.uhf), C.byref(o), C.byref(r), *[_d(out[k]) for k in
                              ("qat", "qsh", "dpat", "qpat", "emo", "P")])
        out.update(energy=r.energy, e_rep=r.e_rep, e_elec=r.e_elec, e_band=r.e_band, e_ts=r.e_ts,
                   e_es2=r.e_es2, e_aes2=r.e_aes2, e_es3=r.e_es3, e_disp=r.e_disp, dipole=np.array(r.dipole[:]),
                   iterations=r.iterations, status=r.status)
        return out

    def singlepoint_gradient(self, mol, **opts):
        """Energy, analytic gradient [nat][3] and virial [3][3] (orc_singlepoint_gradient)."""
        ids = np.ascontiguousarray(mol.id, np.int32); xyz = np.ascontiguousarray(mol.xyz, np.float64)
        o = default_options(**opts)
        r = Result()
        grad, sigma = np.zeros((len(ids), 3)), np.zeros((3, 3))
        lib().orc_singlepoint_gradient(self.h, C.c_int(len(ids)), _i(ids), _d(xyz), C.c_double(mol.charge),
                                       C.c_int(mol.uhf), C.byref(o), C.byref(r), _d(grad), _d(sigma))
        return dict(energy=r.energy, gradient=grad, sigma=sigma, iterations=r.iterations, status=r.status)

    def singlepoint_spin(self, mol, **opts):
        """The singlepoint in the nspin = 2 representation (orc_singlepoint_spin)."""
        ids = np.ascontiguousarray(mol.id, np.int32); xyz = np.ascontiguousarray(mol.xyz, np.float64)
        nat = len(ids); nsh, nao = self.basis_size(ids)
        o = default_options(**opts)
        r = Result()
        out = dict(focc=np.zeros((2, nao)), density=np.zeros((2, nao, nao)), qsh=np.zeros((2, nsh)),
                   qat=np.zeros((2, nat)), dpat=np.zeros((2, nat, 3)), qpat=np.zeros((2, nat, 6)))
        lib().orc_singlepoint_spin(self.h, C.c_int(nat), _i(ids), _d(xyz), C.c_double(mol.charge),
                                   C.c_int(mol.uhf), C.byref(o), C.byref(r),
                                   *[_d(out[k]) for k in ("focc", "density", "qsh", "qat", "dpat", "qpat")])
        out.update(energy=r.energy, iterations=r.iterations, status=r.status)
        return out

    def singlepoint_batch(self, mols, nthreads=1, **opts):
        ids = np.ascontiguousarray(np.concatenate([m.id for m in mols]), np.int32)
        xyz = np.ascontiguousarray(np.concatenate([m.xyz for m in mols]), np.float64)
        aoff = np.zeros(len(mols) + 1, np.int32)
        aoff[1:] = np.cumsum([m.nat for m in mols])
        charge = np.array([m.charge for m in mols], np.float64)
        uhf = np.array([m.uhf for m in mols], np.int32)
        o = default_options(**opts)
        res = (Result * len(mols))()
        lib().orc_singlepoint_batch(self.h, C.c_int(len(mols)), _i(aoff), _i(ids), _d(xyz), _d(charge),
                                    _i(uhf), C.byref(o), C.c_int(nthreads), res)
        return [dict(energy=r.energy, iterations=r.iterations, status=r.status) for r in res]


def kat_multipole_3d(rpj, rpi, aj, ai, lj, li, s1d):
    rpj, rpi, s1d = (np.ascontiguousarray(a, np.float64) for a in (rpj, rpi, s1d))
    lj, li = np.ascontiguousarray(lj, np.int32), np.ascontiguousarray(li, np.int32)
    s3d = C.c_double(); d3d = np.zeros(3); q3d = np.zeros(6)
    lib().orc_multipole_3d(_d(rpj), _d(rpi), C.c_double(aj), C.c_double(ai), _i(lj), _i(li), _d(s1d),
                           C.byref(s3d), _d(d3d), _d(q3d))
    return s3d.value, d3d, q3d


def kat_transform0(lj, li, cart):
    cart = np.ascontiguousarray(cart, np.float64)
    out = np.zeros(25)
    lib().orc_transform0(C.c_int(lj), C.c_int(li), _d(cart), _d(out))
    return out


def kat_gemv(A, x, y, alpha=1.0, beta=0.0, trans=False):
    A, x = np.ascontiguousarray(A, np.float64), np.ascontiguousarray(x, np.float64)
    y = np.array(y, np.float64)
    lib().orc_gemv(C.c_int(A.shape[0]), C.c_int(A.shape[1]), _d(A), _d(x), _d(y), C.c_double(alpha),
                   C.c_double(beta), C.c_int(int(trans)))
    return y
