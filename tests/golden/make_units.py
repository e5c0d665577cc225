"""Generates tests/golden/units_ref.json: the reference's own Python unit
converter (bc/dsmc_unit_converter.py, class DSMC_unit_converter) evaluated on
the conversions the library's Python side restates:

* time_from_si and acceleration_from_si (:63-76), which turn the workloads'
  dt = 1e-11 s and g = 1e9 m/s^2 into the reduced units of the ini files;
* density_from_knudsen_number (:112-116), n = 1 / (sqrt(2) pi d^2 Kn l) in
  m^-3, which sets the Knudsen number of the batched-ensemble geometries
  through their density (l in reduced length units, um).

The converter imports the reference's Python 2 run driver (dsmcconfig) at
module level for nothing the conversions use; an empty stand-in module is
put in its place so the converter loads under Python 3.  Its `dsmc`
argument only has to carry `diam` (reduced, um) for these methods.

    python tests/golden/make_units.py [REFERENCE_PROJECT]
"""
from __future__ import annotations

import importlib.util
import json
import sys
import types
from pathlib import Path

HERE = Path(__file__).resolve().parent
DEFAULT_REF = Path("/root/reference")

KNUDSEN = [0.1, 0.3, 1.0, 3.0, 10.0]
LENGTHS_UM = [0.05, 0.137, 0.4, 1.0, 2.5]
DIAM_UM = 3.66e-4
TIMES_SI = [1e-11, 2.5e-12, 1e-9]
ACCELERATIONS_SI = [1e9, 3.3e8, 1.0]


def load_converter(ref_root: Path):
    path = ref_root / "code" / "base_code" / "dsmc_unit_converter.py"
    sys.modules.setdefault("dsmcconfig", types.ModuleType("dsmcconfig"))
    spec = importlib.util.spec_from_file_location("dsmc_unit_converter", path)
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod.DSMC_unit_converter


def main(argv=None) -> None:
    argv = sys.argv[1:] if argv is None else argv
    ref = Path(argv[0]) if argv else DEFAULT_REF
    conv_cls = load_converter(ref)
    dsmc = types.SimpleNamespace(diam=DIAM_UM)
    uc = conv_cls(dsmc)
    out = {
        "source": "bc/dsmc_unit_converter.py (DSMC_unit_converter)",
        "diam_um": DIAM_UM,
        "time_from_si": [[t, uc.time_from_si(t)] for t in TIMES_SI],
        "acceleration_from_si": [[a, uc.acceleration_from_si(a)] for a in ACCELERATIONS_SI],
        "density_from_knudsen_number": [[kn, l, uc.density_from_knudsen_number(kn, l)]
                                        for kn in KNUDSEN for l in LENGTHS_UM],
    }
    (HERE / "units_ref.json").write_text(json.dumps(out, indent=1) + "\n")
    print("wrote", HERE / "units_ref.json")


if __name__ == "__main__":
    main()
