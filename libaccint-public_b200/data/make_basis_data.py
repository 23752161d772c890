"""Build ``basis_sets.json`` (the basis-set data this package ships) from the
reference's bundled Basis Set Exchange files and its built-in STO-3G table.

Run in a checkout that has the reference tree (argument, else the environment
variable LIBACCINT_REFERENCE, else the default in main()):

    python make_basis_data.py [REFERENCE_ROOT]

Only elements H, C, N, O are kept (the molecules of the benchmark workloads plus
N).  Shell expansion follows the reference's BSE reader
(src/shared/data/bse_json_parser.cpp:27-87): every coefficient column of a
single-l BSE shell becomes its own contracted shell over ALL listed exponents
(zero coefficients included), all-zero columns are skipped, and multi-l (SP)
shells give one shell per l.  The built-in STO-3G (src/shared/data/builtin_basis.cpp)
is parsed from its C++ literals: per element, a list of (l, exponents,
coefficients) in emission order.  So are the reference's built-in auxiliary
(density-fitting) sets of src/shared/data/auxiliary_basis_data.cpp (cc-pVDZ-RI,
cc-pVTZ-RI, def2-SVP-JKFIT, def2-TZVP-JKFIT), stored under their lower-case names.  Coefficients are the raw, un-normalized
contraction coefficients; normalization happens when a basis is built.
"""
import json
import os
import re
import sys

ELEMENTS = {"1": "H", "6": "C", "7": "N", "8": "O"}
BSE_FILES = ["sto-3g", "6-31g", "cc-pvdz", "cc-pvtz", "cc-pvqz", "aug-cc-pvdz", "aug-cc-pvtz"]


def expand_bse_element(el):
    shells = []
    for sh in el.get("electron_shells", []):
        exps = [float(x) for x in sh["exponents"]]
        ams = [int(a) for a in sh["angular_momentum"]]
        cols = [[float(c) for c in col] for col in sh["coefficients"]]
        if len(ams) == 1:
            for col in cols:
                if any(c != 0.0 for c in col):
                    shells.append([ams[0], exps, col])
        else:
            for am, col in zip(ams, cols):
                if any(c != 0.0 for c in col):
                    shells.append([am, exps, col])
    return shells


def parse_builtin_sto3g(path):
    src = open(path).read()
    out = {}
    names = {"hydrogen": "H", "carbon": "C", "nitrogen": "N", "oxygen": "O", "fluorine": "F"}
    for fn, body in re.findall(r"void add_(\w+)_sto3g\([^)]*\)\s*\{(.*?)\n\}", src, re.S):
        shells = []
        for am, e, c in re.findall(
                r"emplace_back\(\s*(\d+),\s*center,\s*std::vector<Real>\{([^}]*)\},\s*"
                r"std::vector<Real>\{([^}]*)\}", body, re.S):
            shells.append([int(am), [float(x) for x in e.split(",")],
                           [float(x) for x in c.split(",")]])
        if fn in names and names[fn] in ELEMENTS.values():
            out[names[fn]] = shells
    return out


def parse_builtin_aux(path):
    src = open(path).read()
    names = {"hydrogen": "H", "carbon": "C", "nitrogen": "N", "oxygen": "O"}
    sets = {"cc_pvdz_ri": "cc-pvdz-ri", "cc_pvtz_ri": "cc-pvtz-ri", "def2_svp_jkfit": "def2-svp-jkfit",
            "def2_tzvp_jkfit": "def2-tzvp-jkfit"}
    out = {v: {} for v in sets.values()}
    for fn, body in re.findall(r"std::vector<AuxShellData> (\w+)\(\)\s*\{(.*?)\n\}", src, re.S):
        for prefix, key in sets.items():
            if fn.startswith(prefix + "_") and fn[len(prefix) + 1:] in names:
                shells = []
                for am, e, c in re.findall(r"\{\s*(\d+),\s*\{([^}]*)\},\s*\{([^}]*)\}\s*\}", body):
                    shells.append([int(am), [float(x) for x in e.split(",")], [float(x) for x in c.split(",")]])
                out[key][names[fn[len(prefix) + 1:]]] = shells
    return out


def main():
    ref = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("LIBACCINT_REFERENCE", "/root/reference")
    data = {}
    for name in BSE_FILES:
        j = json.load(open(os.path.join(ref, "share", "basis_sets", name + ".json")))
        data[name] = {sym: expand_bse_element(j["elements"][z])
                      for z, sym in ELEMENTS.items() if z in j["elements"]}
    data["sto-3g-builtin"] = parse_builtin_sto3g(
        os.path.join(ref, "src", "shared", "data", "builtin_basis.cpp"))
    data.update(parse_builtin_aux(os.path.join(ref, "src", "shared", "data", "auxiliary_basis_data.cpp")))
    here = os.path.dirname(os.path.abspath(__file__))
    with open(os.path.join(here, "basis_sets.json"), "w") as f:
        json.dump({"source": "reference share/basis_sets (Basis Set Exchange) and "
                             "src/shared/data/builtin_basis.cpp and auxiliary_basis_data.cpp",
                   "basis_sets": data}, f, separators=(",", ":"))


if __name__ == "__main__":
    main()
