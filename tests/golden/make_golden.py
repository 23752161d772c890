"""Generate the committed golden fixtures of tests/golden/ (run in a checkout
that has the reference tree and oracle/_ref built: ``make -C oracle``).

Fixtures and their provenance:

* boys_mpmath.npz     -- tests/data/boys_reference.json of the reference (mpmath,
                         50 digits): T points and F_0..F_n(T).
* rys_refgen.npz      -- tests/data/rys_reference.json (the reference's own
                         rys_compute output; a regression fixture, not independent).
* water1_augccpvtz.npz-- tests/data/reference/water_1_aug_cc_pVTZ.json (PySCF 2.11,
                         cart=True): geometry, density, J, K, sampled ERIs, shell
                         table.  Checked at 1e-7 by the reference's own
                         test_water_cluster_validation.cpp:454-495.
* <workload>_ref.npz  -- J/K of the UNMODIFIED reference, Engine::compute(coulomb,
                         FockBuilder) (full N^4, no screening), for the seeded
                         workloads h2o8_sto3g (config 0: built-in STO-3G, 8 waters),
                         h2o2_ccpvdz and h2o1_ccpvqz (s..g shells, every class up
                         to (gg|gg); about 150 s on 8 cores, option "refqz"), plus
                         the density used.
* one_electron_sto3g.npz -- tests/integration/test_one_electron.cpp of the reference
                         (PySCF cart=True values written into the test): the H2 and
                         H2O STO-3G shells, point charges and S, T, V matrices; and
                         tests/integration/test_hf_energy.cpp: RHF total energies of
                         H2, H2O and CH4 with the built-in STO-3G (PySCF) and the H2O
                         nuclear repulsion.  Parsed from the test sources as text.
* eri_ccpvqz_samples.npz -- per-integral values of sampled shell quartets of all
                         angular-momentum classes present in an H2O + CH4 pair with
                         cc-pVQZ (up to g): the reference's compute_eri and the
                         binary128-root restatement oracle side by side.
"""
import importlib
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
# reference checkout: argument, else $LIBACCINT_REFERENCE, else the default below
REF = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("LIBACCINT_REFERENCE", "/root/reference")
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))
import oracle  # noqa: E402

lai = importlib.import_module("libaccint-public_b200")


def boys():
    d = json.load(open(os.path.join(REF, "tests", "data", "boys_reference.json")))
    T = np.array([p["T"] for p in d["test_points"]])
    nmax = min(len(p["values"]) for p in d["test_points"])
    F = np.array([p["values"][:nmax] for p in d["test_points"]])
    np.savez_compressed(os.path.join(HERE, "boys_mpmath.npz"), T=T, F=F)


def rys():
    d = json.load(open(os.path.join(REF, "tests", "data", "rys_reference.json")))["rys_quadrature"]
    out = {}
    for n, per_t in d["data"].items():
        T = np.array([float(t) for t in per_t])
        out[f"n{n}_T"] = T
        out[f"n{n}_roots"] = np.array([[float(x) for x in v["roots"]] for v in per_t.values()])
        out[f"n{n}_weights"] = np.array([[float(x) for x in v["weights"]] for v in per_t.values()])
    np.savez_compressed(os.path.join(HERE, "rys_refgen.npz"), **out)


def water1():
    d = json.load(open(os.path.join(REF, "tests", "data", "reference", "water_1_aug_cc_pVTZ.json")))
    n = d["n_basis"]
    xyz = np.array(d["molecule"]["geometry_bohr"])
    D = np.array(d["density_matrix"]["matrix"]).reshape(n, n)
    J = np.array(d["fock_from_density"]["coulomb_matrix"]).reshape(n, n)
    K = np.array(d["fock_from_density"]["exchange_matrix"]).reshape(n, n)
    idx = np.array([e["indices"] for e in d["sampled_eri"]], dtype=np.int64)
    val = np.array([e["value"] for e in d["sampled_eri"]])
    shells = np.array([[s["atom"], s["angular_momentum"], s["n_primitives"], s["ao_start"]]
                       for s in d["shells"]], dtype=np.int64)
    np.savez_compressed(os.path.join(HERE, "water1_augccpvtz.npz"), xyz=xyz, Z=np.array([8, 1, 1]),
                        D=D, J=J, K=K, eri_idx=idx, eri_val=val, shells=shells,
                        rhf_energy=d["rhf"]["total_energy"])


def ref_jk(name):
    w = lai.workloads.make(name)
    if name.endswith("sto3g"):
        R = oracle.RefBasis(builtin_sto3g=(w.Z, w.xyz))
    else:
        R = oracle.RefBasis(w.basis)
    assert R.nbf == w.nbf
    J, K, t = R.jk_full(w.D, 0)
    print(name, "reference full J/K", t, "s")
    np.savez_compressed(os.path.join(HERE, name + "_ref.npz"), Z=w.Z, xyz=w.xyz, D=w.D, J=J, K=K)


def norm_ccpvqz():
    """Normalized contraction coefficients of the reference Shell ctor (CH4 cc-pVQZ)."""
    Z = np.array([6, 1], dtype=np.int32)
    xyz = np.array([[0.0, 0.0, 0.0], [1.2, 0.9, -1.1]])
    b = lai.BasisSet.from_atoms(Z, xyz, "cc-pvqz")
    R = oracle.RefBasis(b)
    coefs = np.concatenate([R.shell_info(i)[3] for i in range(R.nshell)])
    np.savez_compressed(os.path.join(HERE, "norm_ccpvqz_ref.npz"), Z=Z, xyz=xyz, coefs=coefs)


def eri_samples(nsample=400, seed=3):
    """Sampled quartets of a water + methane pair in cc-pVQZ (l up to g on C)."""
    Zw, xw = lai.molecules.water_cluster((1, 1, 1), np.random.default_rng(11))
    Zc = np.array([6, 1, 1, 1, 1], dtype=np.int32)
    a = 1.18
    xc = np.array([[0, 0, 0], [a, a, a], [-a, -a, a], [-a, a, -a], [a, -a, -a]], dtype=float) + [4.0, 1.0, 0.5]
    Z = np.concatenate([Zw, Zc])
    xyz = np.concatenate([xw, xc])
    b = lai.BasisSet.from_atoms(Z, xyz, "cc-pvqz")
    R = oracle.RefBasis(b)
    rng = np.random.default_rng(seed)
    ls = np.array([s.l for s in b.shells])
    # cover every (la,lb,lc,ld) class multiset present, then random extras
    quartets = []
    seen = set()
    for _ in range(200000):
        q = rng.integers(0, b.n_shells, 4)
        key = tuple(ls[q])
        if key not in seen:
            seen.add(key)
            quartets.append(q)
        if len(quartets) >= nsample:
            break
    # keep at most 40 integrals per quartet (random flat indices) to stay small
    rows, flat, ref_vals, orc_vals = [], [], [], []
    for qi, q in enumerate(quartets):
        shape = tuple((ls[x] + 1) * (ls[x] + 2) // 2 for x in q)
        r = R.quartet(*map(int, q), shape).ravel()
        o = oracle.orc_quartet(b, *map(int, q)).ravel()
        pick = np.sort(rng.choice(r.size, size=min(40, r.size), replace=False))
        rows += [qi] * len(pick)
        flat += list(pick)
        ref_vals.append(r[pick])
        orc_vals.append(o[pick])
    np.savez_compressed(os.path.join(HERE, "eri_ccpvqz_samples.npz"), Z=Z, xyz=xyz,
                        quartets=np.array(quartets, dtype=np.int64), row=np.array(rows),
                        flat=np.array(flat), ref=np.concatenate(ref_vals), orc=np.concatenate(orc_vals))


def _floats(txt):
    import re
    return [float(x) for x in re.findall(r"[-+]?\d+\.\d*(?:[eE][-+]?\d+)?", txt)]


def one_electron():
    import re
    src = open(os.path.join(REF, "tests/integration/test_one_electron.cpp")).read()
    out = {}
    for arr in ("H2_S_REF", "H2_T_REF", "H2_V_REF", "H2O_S_REF", "H2O_T_REF", "H2O_V_REF"):
        m = re.search(r"constexpr Real %s\[(\d+)\] = \{(.*?)\};" % arr, src, re.S)
        body = "\n".join(line.split("//")[0] for line in m.group(2).splitlines())
        vals = _floats(body)
        assert len(vals) == int(m.group(1)), arr
        n = int(round(len(vals) ** 0.5))
        out[arr] = np.array(vals).reshape(n, n)
    # shells of make_h2_sto3g / make_h2o_sto3g
    vecs = {k: _floats(v) for k, v in re.findall(r"std::vector<Real> (\w+) = \{([^}]*)\};", src)}
    for name, fn in (("h2", "make_h2_sto3g"), ("h2o", "make_h2o_sto3g")):
        body = src[src.index("BasisSet %s()" % fn):]
        body = body[:body.index("return BasisSet")]
        pts = {k: _floats(v) for k, v in re.findall(r"Point3D (\w+)\{([^}]*)\};", body)}
        ls, ctr, ex, co, npr = [], [], [], [], []
        for m in re.finditer(r"Shell (\w+)\((\d),\s*(\w+),\s*(\{[^}]*\}|\w+),\s*(\{[^}]*\}|\w+)\);", body):
            e = _floats(m.group(4)) if m.group(4).startswith("{") else vecs[m.group(4)]
            c = _floats(m.group(5)) if m.group(5).startswith("{") else vecs[m.group(5)]
            ls.append(int(m.group(2)))
            ctr.append(pts[m.group(3)])
            ex += e
            co += c
            npr.append(len(e))
        out[name + "_l"] = np.array(ls, dtype=np.int32)
        out[name + "_center"] = np.array(ctr)
        out[name + "_nprim"] = np.array(npr, dtype=np.int32)
        out[name + "_exps"] = np.array(ex)
        out[name + "_coefs"] = np.array(co)
        cb = src[src.index("PointChargeParams %s_charges()" % fn.replace("_sto3g", "").replace("make_", "make_")):]
        cb = cb[:cb.index("return charges")]
        xyz = [_floats(re.search(r"charges\.%s = \{([^}]*)\}" % k, cb).group(1)) for k in "xyz"]
        out[name + "_charge_xyz"] = np.array(xyz).T.copy()
        out[name + "_charge_q"] = np.array(_floats(re.search(r"charges\.charge = \{([^}]*)\}", cb).group(1)))
    hf = open(os.path.join(REF, "tests/integration/test_hf_energy.cpp")).read()
    for test, key in (("H2O_STO3G", "hf_h2o"), ("H2_STO3G", "hf_h2"), ("CH4_STO3G", "hf_ch4")):
        body = hf[hf.index("TEST(HFEnergyTest, %s)" % test):]
        body = body[:body.index("EXPECT_NEAR")]
        consts = dict((k, float(v)) for k, v in re.findall(r"constexpr Real (\w+) = ([-+0-9.eE]+);", body))
        atoms = re.findall(r"\{(\d+),\s*\{([^}]*)\}\}", body)
        Z, xyz = [], []
        for z, r in atoms:
            comps = []
            for tok in r.split(","):
                tok = tok.strip()
                sgn = -1.0 if tok.startswith("-") else 1.0
                tok = tok.lstrip("+-")
                comps.append(sgn * (consts[tok] if tok in consts else float(tok)))
            Z.append(int(z))
            xyz.append(comps)
        out[key + "_Z"] = np.array(Z, dtype=np.int32)
        out[key + "_xyz"] = np.array(xyz)
        out[key + "_energy"] = np.array(consts["REF_ENERGY"])
        out[key + "_nelec"] = np.array(sum(Z))
    m = re.search(r"EXPECT_NEAR\(E_nuc, ([-+0-9.eE]+)", hf)
    out["h2o_enuc"] = np.array(float(m.group(1)))
    np.savez_compressed(os.path.join(HERE, "one_electron_sto3g.npz"), **out)


if __name__ == "__main__":
    only = sys.argv[2:] if len(sys.argv) > 2 else ["boys", "rys", "water1", "ref", "eri", "one"]
    if "one" in only:
        one_electron()
    if "boys" in only:
        boys()
    if "rys" in only:
        rys()
    if "water1" in only:
        water1()
    if "ref" in only:
        ref_jk("h2o8_sto3g")
        ref_jk("h2o2_sto3g")
        ref_jk("h2o2_ccpvdz")
        norm_ccpvqz()
    if "refqz" in only:
        ref_jk("h2o1_ccpvqz")
    if "eri" in only:
        eri_samples()
