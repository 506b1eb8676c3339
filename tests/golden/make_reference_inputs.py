"""Writes tests/golden/reference_inputs.json from the reference's own input files.

The polarization path's parameters and settings come from files the reference
ships: the AMOEBA water parameter files (v1.2/params/water03.prm, water.prm)
and the keyword files of its 288,000-atom water benchmark "pond"
(v1.2/example/pond.key, v1.1v/example/pond/pond.key).  This script parses them
with the package's own Tinker reader (tinker_io.read_params) and stores the
parsed values, so that the CPU tests can compare the built-in parameter table
(params.py) and the benchmark workload with what the reference reads, on a
machine without the reference tree.

Run from the repository root, with the reference checked out at REF (default
/root/reference):  python tests/golden/make_reference_inputs.py [REF]
"""
import json
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
OUT = os.path.join(HERE, "reference_inputs.json")

# files read, relative to the reference root
FILES = {
    "water03": "v1.2/params/water03.prm",
    "water": "v1.2/params/water.prm",
    "pond_v12": "v1.2/example/pond.key",
    "pond_v11": "v1.1v/example/pond/pond.key",
    "water_v11": "v1.1v/params/water.prm",
}
# the keywords of the path that the key files set
KEYWORDS = ("EWALD", "EWALD-CUTOFF", "VDW-CUTOFF", "PME-GRID", "POLAR-EPS", "POLAR-ALG", "X-AXIS",
            "A-AXIS", "NEIGHBOR-LIST", "POLARIZATION", "FORCEFIELD", "PARAMETERS")


def _tinker_io():
    sys.path.insert(0, ROOT)
    from tests.conftest import load_package
    load_package()
    from tinker_hp_b200 import tinker_io
    return tinker_io


def parsed(ref):
    T = _tinker_io()
    path = {k: os.path.join(ref, v) for k, v in FILES.items()}

    def param_set(ps):
        return {
            "multipoles": [{"type": m.k, "kz": m.kz, "kx": m.kx, "ky": m.ky, "frame": m.frame,
                            "values": list(m.values)} for m in ps.multipoles],
            "polarize": {str(t): {"polarity": v[0], "thole": v[1], "group": list(v[3])}
                         for t, v in sorted(ps.polarize.items())},
            "scales": {k: list(v) for k, v in sorted(ps.scales.items())},
            "vdw": {str(c): list(v) for c, v in sorted(ps.vdw.items())},
            "vdw_scale": list(ps.v_scale),
            "keywords": {k: ps.keywords[k] for k in KEYWORDS if k in ps.keywords},
        }

    out = {"files": FILES}
    out["water03"] = param_set(T.read_params(prm_path=path["water03"]))
    out["water"] = param_set(T.read_params(prm_path=path["water"]))
    # pond.key (v1.2) names its parameter file relative to itself
    out["pond_v12"] = param_set(T.read_params(key_path=path["pond_v12"]))
    # pond.key (v1.1v) names "water", found by its run script in ../../params
    out["pond_v11"] = param_set(T.read_params(key_path=path["pond_v11"], prm_path=path["water_v11"]))
    return out


def main():
    ref = sys.argv[1] if len(sys.argv) > 1 else "/root/reference"
    data = parsed(ref)
    with open(OUT, "w") as f:
        json.dump(data, f, indent=1, sort_keys=True)
        f.write("\n")
    print("wrote", OUT)


if __name__ == "__main__":
    main()
