"""Generate the golden fixtures in this folder from the reference's own sources.

Runs only where the reference tree is mounted (it builds and loads
oracle/_ref/libscp3ref.so, compiled from the reference's unmodified sources by
oracle/Makefile).  The committed .npz files are what the tests read; nothing
here runs on a GPU box.

    python tests/golden/make_golden.py            # writes tests/golden/*.npz

Fixtures:
  sobol_ref.npz   i8_sobol uniforms (sobol.cpp:14198-27868) and std_normal draws
                  (sobol.cpp:28706-28713), from index 0 and from the default skip 2^30
                  (SCP3.cpp:48), 66 dimensions.
  pes_ref.npz     qTIP4P/f and TTM3-F energies (qtip4pf.cpp:190-286, ttm3f.cpp:92-321)
                  on the test-potentials.cpp:14-33 prism, relaxed dimer/prism, random
                  3- and 4-water clusters and seeded perturbations of each.
  hbuild_ref.npz  the -G sample loop (SCP3.cpp:187-232 with get_bra + dsyr2k,
                  ScaledMatrixElements.cpp:870-971) for small dimer/hexamer bases,
                  with the normal-mode inputs it used.
  stein_ref.npz   the gradient path: every formula of TripleExcitations.h (the
                  reference's gradient estimator, oracle/_ref/libscp3ref_stein.so)
                  on seeded data; qTIP4P/f gradients (qtip4pf.cpp:252-397) on the
                  pes_ref geometries; and a dimer matrix (N2 = 12, N3 = 4) summed
                  from the reference's formulas over samples whose V and dV/dq
                  come from the reference's potential (SCP3.cpp:205-223).

    python tests/golden/make_golden.py stein      # only stein_ref.npz
"""
import os
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

import oracle  # noqa: E402
from scp3_b200 import clusters, constants as C, modes  # noqa: E402

OUT = os.path.dirname(os.path.abspath(__file__))
REF = os.environ.get("SCP3_REFERENCE")

# test-potentials.cpp:14-33, O H H order, Angstrom
PRISM_TP = np.array([
    -1.501133590, -0.197346710, 1.441262950, -2.000985830, -0.388094000, 2.232286820,
    -0.613018210, -0.604501640, 1.565741520, -1.738921070, -0.356671650, -1.311647220,
    -2.485655290, -0.756663570, -1.757003500, -1.883593590, -0.495826200, -0.359467970,
    -0.590049110, 2.045369740, -0.113997110, -1.009913650, 1.627267800, -0.873288670,
    -0.961441910, 1.549440890, 0.629166980, 0.999999910, -1.179514770, 1.454043080,
    1.550433810, -0.395916830, 1.334139300, 1.004009200, -1.558530670, 0.559262460,
    0.982946210, -1.411538550, -1.350690300, 1.478885410, -0.585694520, -1.278498130,
    0.076249970, -1.127406420, -1.530339410, 1.967206930, 1.048112740, -0.137872390,
    2.659992820, 1.698771500, -0.239214400, 1.124990980, 1.547180090, -0.146635510])


def ref_energy(L, fn):
    def f(X):
        X = np.atleast_2d(X)
        return np.array([getattr(L, fn)(x.size // 9, oracle._dp(np.ascontiguousarray(x))) for x in X])
    return f


def gen_sobol(L):
    import ctypes
    dims = 66
    seed = ctypes.c_longlong(0)
    u0 = np.zeros((64, dims))
    for k in range(64):
        L.ref_i8_sobol(dims, ctypes.byref(seed), oracle._dp(u0[k]))
    seed = ctypes.c_longlong(1 << 30)
    t = time.time()
    u30 = np.zeros((8, dims))
    for k in range(8):
        L.ref_i8_sobol(dims, ctypes.byref(seed), oracle._dp(u30[k]))
    print("skip walk %.1fs" % (time.time() - t))
    seed = ctypes.c_longlong(1 << 30)
    n30 = np.zeros((16, 48))
    for k in range(16):
        L.ref_std_normal(48, ctypes.byref(seed), oracle._dp(n30[k]))
    np.savez_compressed(os.path.join(OUT, "sobol_ref.npz"), u_from0=u0, u_from2_30=u30, std_normal48_from2_30=n30)


def gen_pes(L):
    rng = np.random.default_rng(2024)
    eq = ref_energy(L, "ref_qtip4pf_energy")
    dimer, _, _, _ = clusters.relax(eq, clusters.dimer(), maxiter=400)
    prism, _, _, _ = clusters.relax(eq, clusters.prism(), maxiter=400)
    bases = [PRISM_TP, dimer, prism, clusters.random_cluster(3, 7), clusters.random_cluster(4, 11),
             clusters.water().ravel()]
    geoms = []
    for b in bases:
        geoms.append(b)
        for _ in range(6):
            geoms.append(b + rng.normal(scale=0.05, size=b.size))
    names = []
    eq_out, et_out = [], []
    et = ref_energy(L, "ref_ttm3f_energy")
    for g in geoms:
        eq_out.append(eq(g)[0])
        et_out.append(et(g)[0])
        names.append(g.size // 9)
    obj = np.empty(len(geoms), dtype=object)
    obj[:] = geoms
    np.savez_compressed(os.path.join(OUT, "pes_ref.npz"), geoms=obj, nw=np.array(names),
                        e_qtip4pf=np.array(eq_out), e_ttm3f=np.array(et_out), allow_pickle=True)
    return dimer, prism


def setup_modes(L, x):
    eq = ref_energy(L, "ref_qtip4pf_energy")
    nw = x.size // 9
    mass = np.tile(np.repeat([C.Omass, C.Hmass, C.Hmass], 3), nw)
    H, x0 = clusters.hessian(eq, x, mass)
    omega, MUa, _ = modes.normal_modes(H, mass)
    return x0, MUa, omega


def gen_hbuild(L, dimer, prism):
    cases = {}
    specs = [
        # name, geometry, pes, modes, N2, N3, nsamples, block, scramble seed (None = reference Sobol from 2^30)
        ("dimer_qtip4pf", dimer, 0, None, 12, 4, 2048, 256, 0x5C3),
        ("dimer_qtip4pf_unscrambled", dimer, 0, None, 12, 0, 1024, 256, None),
        ("hexamer_qtip4pf", prism, 0, None, 10, 6, 512, 256, 0x5C3),
        ("hexamer_qtip4pf_modesel", prism, 0, np.r_[0:8, 20:30, 40:48], 8, 3, 256, 128, 77),
        ("dimer_ttm3f", dimer, 1, None, 12, 3, 512, 256, 0x5C3),
        ("hexamer_ttm3f", prism, 1, None, 6, 4, 256, 128, 0x5C3),
    ]
    for name, x, pes, sel, n2, n3, ns, block, sseed in specs:
        x0, MUa, omega = setup_modes(L, x)
        nw = x.size // 9
        nm0 = omega.size
        sel = np.arange(nm0, dtype=np.int32) if sel is None else np.asarray(sel, dtype=np.int32)
        if sseed is None:
            normals = oracle.std_normals(nm0, 1 << 30, ns)
        else:
            normals = oracle.std_normals(nm0, 0, ns, scramble_seed=sseed)
        M, _, _ = oracle.ref_hbuild(pes, nw, x0, MUa, omega, sel, n2, n3, ns, block, normals=normals)
        iu = np.triu_indices(M.shape[0])
        cases[name] = dict(x0=x0, MUa=MUa, omega=omega, modes=sel, pes=pes, nw=nw, n2=n2, n3=n3,
                           nsamples=ns, block=block, scramble_seed=-1 if sseed is None else sseed,
                           index0=(1 << 30) if sseed is None else 0, M_upper=M.T[iu[1], iu[0]])
        print(name, M.shape, "done")
    flat = {}
    for name, d in cases.items():
        for k, v in d.items():
            flat[name + "__" + k] = np.asarray(v)
    np.savez_compressed(os.path.join(OUT, "hbuild_ref.npz"), **flat)


def parse_formula(name, params):
    """TripleExcitations.h names a formula by its bra and ket, e.g.
    m2_n1_f_k1_l1_j1(m, n, k, l, j) = <2_m 1_n | V | 1_k 1_l 1_j>: per side a
    list of (parameter index, level)."""
    bra, ket = name.split("f_") if name.startswith("f_") is False else ("", name[2:])
    if not name.startswith("f_"):
        bra, ket = name.split("_f_")
    side = lambda t: [(params.index(tok[0]), int(tok[1])) for tok in t.split("_") if tok]
    return side(bra), side(ket)


def ref_stein_lib():
    import ctypes
    Ls = ctypes.CDLL(os.path.join(ROOT, "oracle", "_ref", "libscp3ref_stein.so"))
    Ls.ref_stein_name.restype = ctypes.c_char_p
    Ls.ref_stein_params.restype = ctypes.c_char_p
    dp = ctypes.POINTER(ctypes.c_double)
    Ls.ref_stein_eval.restype = ctypes.c_double
    Ls.ref_stein_eval.argtypes = [ctypes.c_int, dp, dp, dp, ctypes.c_int, ctypes.POINTER(ctypes.c_int)]
    names = [Ls.ref_stein_name(i).decode() for i in range(Ls.ref_stein_count())]
    params = [Ls.ref_stein_params(i).decode().split(",") for i in range(Ls.ref_stein_count())]
    return Ls, names, params


def ref_stein_eval(Ls, i, args, qT, V, VqT):
    import ctypes
    dp = ctypes.POINTER(ctypes.c_double)
    a = np.asarray(args, dtype=np.int32)
    return Ls.ref_stein_eval(i, qT.ctypes.data_as(dp), V.ctypes.data_as(dp), VqT.ctypes.data_as(dp), V.size,
                             a.ctypes.data_as(ctypes.POINTER(ctypes.c_int)))


def gen_stein(L, dimer):
    import ctypes
    import itertools
    Ls, names, params = ref_stein_lib()
    rng = np.random.default_rng(2024)
    nm, n = 10, 64
    q = rng.normal(scale=np.sqrt(0.5), size=(n, nm))
    V = rng.normal(size=n)
    Vq = rng.normal(size=(n, nm))
    qT, VqT = np.ascontiguousarray(q.T), np.ascontiguousarray(Vq.T)
    args = np.full((len(names), 6), -1, dtype=np.int32)
    vals = np.zeros(len(names))
    for i, (nmx, pr) in enumerate(zip(names, params)):
        a = rng.choice(nm, size=len(pr), replace=False)
        args[i, :len(pr)] = a
        vals[i] = ref_stein_eval(Ls, i, a, qT, V, VqT)
    # qTIP4P/f gradients of the reference on the pes_ref geometries
    dp = ctypes.POINTER(ctypes.c_double)
    L.ref_qtip4pf_energy_grad.restype = ctypes.c_double
    L.ref_qtip4pf_energy_grad.argtypes = [ctypes.c_int, dp, dp]
    z = np.load(os.path.join(OUT, "pes_ref.npz"), allow_pickle=True)
    L.ref_ttm3f_energy_grad.restype = ctypes.c_double
    L.ref_ttm3f_energy_grad.argtypes = [ctypes.c_int, dp, dp]
    grads, grads_t, e_t = [], [], []
    for x in z["geoms"]:
        x = np.ascontiguousarray(x, dtype=np.float64)
        g = np.zeros(x.size)
        L.ref_qtip4pf_energy_grad(x.size // 9, x.ctypes.data_as(dp), g.ctypes.data_as(dp))
        grads.append(g)
        # TTM3-F E+g twice: its dipole iteration starts from the previous call's field
        # (ttm3f.cpp:344-345 zeroes Efd/Efq/phi/dM here, so one call suffices; two agree)
        g = np.zeros(x.size)
        L.ref_ttm3f_energy_grad(x.size // 9, x.ctypes.data_as(dp), g.ctypes.data_as(dp))
        e_t.append(L.ref_ttm3f_energy_grad(x.size // 9, x.ctypes.data_as(dp), g.ctypes.data_as(dp)))
        grads_t.append(g)
    out = dict(names=np.array(names), params=np.array([",".join(p) for p in params]), args=args, values=vals,
               q=q, V=V, Vq=Vq, pes_geoms_grad=np.array(grads, dtype=object),
               pes_geoms_grad_ttm3f=np.array(grads_t, dtype=object), pes_geoms_e_ttm3f=np.array(e_t))
    x0, MUa, omega = setup_modes(L, dimer)
    for tag, fn in (("dimer", L.ref_qtip4pf_energy_grad), ("dimer_ttm3f", L.ref_ttm3f_energy_grad)):
        n2, n3, ns, sseed = 12, 4, 256, 0x5C3
        qs, Vs, Vqs, Mu = stein_matrix(Ls, names, params, fn, x0, MUa, omega, n2, n3, ns, sseed)
        out.update({tag + "_x0": x0, tag + "_MUa": MUa, tag + "_omega": omega, tag + "_n2": n2, tag + "_n3": n3,
                    tag + "_nsamples": ns, tag + "_scramble_seed": sseed, tag + "_q": qs, tag + "_V": Vs,
                    tag + "_Vq": Vqs, tag + "_M_upper": Mu})
    np.savez_compressed(os.path.join(OUT, "stein_ref.npz"), **out)


def stein_matrix(Ls, names, params, egrad, x0, MUa, omega, n2, n3, ns, sseed):
    """A gradient-path matrix from the reference: V and dV/dq from the
    reference's E+g operator (SCP3.cpp:205-223) and every upper element from
    the reference formula for its bra and ket."""
    import ctypes
    import itertools
    dp = ctypes.POINTER(ctypes.c_double)
    nm0 = omega.size
    normals = oracle.std_normals(nm0, 0, ns, scramble_seed=sseed)
    bohr, kcal = C.bohr, C.autokcalpmol
    qs = normals / np.sqrt(2.0)
    Vs = np.zeros(ns)
    Vqs = np.zeros((ns, nm0))
    for s in range(ns):
        r = np.ascontiguousarray(bohr * (x0 + MUa @ qs[s]))
        g = np.zeros(r.size)
        egrad(r.size // 9, r.ctypes.data_as(dp), g.ctypes.data_as(dp))
        e = egrad(r.size // 9, r.ctypes.data_as(dp), g.ctypes.data_as(dp)) / kcal
        Vs[s] = e - 0.5 * np.dot(qs[s], omega * qs[s])
        Vqs[s] = MUa.T @ (g * bohr / kcal) - omega * qs[s]
    nb = oracle.basis_size(nm0, n2, n3)
    funcs = [oracle.basis_modes(nm0, n2, n3, R) for R in range(nb)]
    parsed = [parse_formula(nmx, pr) for nmx, pr in zip(names, params)]
    qT, VqT = np.ascontiguousarray(qs.T), np.ascontiguousarray(Vqs.T)
    Mu = np.zeros(nb * (nb + 1) // 2)
    k = 0
    used = set()
    for C_ in range(nb):
        for R in range(C_ + 1):
            if R == 0 and C_ == 0:
                Mu[k] = Vs.sum()            # M(0,0) += sum(V), ScaledMatrixElements.cpp:711
                k += 1
                continue
            hit = None
            # a formula names <bra|V|ket>; the estimate is symmetric, so either
            # function of the pair may be its bra (the loops of
            # ScaledMatrixElements.cpp:102-702 use both orders)
            for i, (pb, pk), (bra, ket) in ((i, pp, bk) for bk in ((funcs[R], funcs[C_]), (funcs[C_], funcs[R]))
                                            for i, pp in enumerate(parsed)):
                if len(pb) != len(bra) or len(pk) != len(ket):
                    continue
                for perm_b in itertools.permutations(range(len(bra))):
                    ok = all(bra[perm_b[t]][1] == pb[t][1] for t in range(len(pb)))
                    if not ok:
                        continue
                    amap = {pb[t][0]: bra[perm_b[t]][0] for t in range(len(pb))}
                    for perm_k in itertools.permutations(range(len(ket))):
                        a2 = dict(amap)
                        good = True
                        for t in range(len(pk)):
                            md, lv = ket[perm_k[t]]
                            if lv != pk[t][1] or a2.get(pk[t][0], md) != md:
                                good = False
                                break
                            a2[pk[t][0]] = md
                        if good and len(set(a2.values())) == len(a2) and len(a2) == len(params[i]):
                            hit = (i, [a2[j] for j in range(len(params[i]))])
                            break
                    if hit:
                        break
                if hit:
                    break
            if hit is None:
                raise RuntimeError("no formula for <%s|V|%s>" % (funcs[R], funcs[C_]))
            used.add(hit[0])
            Mu[k] = ref_stein_eval(Ls, hit[0], hit[1], qT, Vs, VqT)
            k += 1
    print("stein: %d formulas, %d used by the dimer matrix" % (len(names), len(used)))
    return qs, Vs, Vqs, Mu


def main():
    if not REF:
        sys.exit("set SCP3_REFERENCE to the reference tree's root")
    oracle.build(REF)
    L = oracle.ref_lib()
    if sys.argv[1:] == ["stein"]:
        z = np.load(os.path.join(OUT, "pes_ref.npz"), allow_pickle=True)
        gen_stein(L, np.asarray(z["geoms"][7], dtype=np.float64))   # the relaxed dimer (gen_pes bases[1])
        return
    gen_sobol(L)
    dimer, prism = gen_pes(L)
    gen_hbuild(L, dimer, prism)
    gen_stein(L, dimer)


if __name__ == "__main__":
    main()
