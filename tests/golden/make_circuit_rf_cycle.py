"""Generates circuit_rf_cycle.npz: the RF circuit waveform of the reference's own
circuit_rf benchmark run, computed by the reference's circuit model here.

    python tests/golden/make_circuit_rf_cycle.py /path/to/reference
    (or TRENCH01_REFERENCE=/path/to/reference python tests/golden/make_circuit_rf_cycle.py)

The run is the one documented in the reference's docs/rf_cycle_validation.json
(3000 batches of 3000 ions + 3000 electrons on a 120 x 560 grid, pulsed 5 kV
bias at 400 kHz, circuit_rf field mode).  In circuit_rf mode the reference's
run() asks the circuit for the waveform only (trench_charging_2d.py:1074,
include_ied=False: ions enter at Te/2 and are accelerated in flight), so the
file holds that waveform -- the electrode potentials over one period -- and the
parameters.  The circuit model is the reference's CPU code and an input to the
charging step; the benchmark reads this file instead of running it.
"""
import json
import sys
from dataclasses import asdict, replace
from pathlib import Path

import numpy as np

sys.path.insert(0, str(Path(__file__).resolve().parent))
from make_golden import import_reference, reference_dir, save  # noqa: E402


def main(ref):
    T, _ = import_reference(ref)
    import plasma_circuit as PC
    doc = json.loads((Path(ref) / "docs" / "rf_cycle_validation.json").read_text())
    base = T.Params()
    p = replace(base, **{k: v for k, v in doc["params"].items() if hasattr(base, k)})
    c = PC.solve_circuit(p, include_ied=False)
    save("circuit_rf_cycle.npz", params=json.dumps(asdict(p)), t=c["t"], uw=c["uw"], um=c["um"], up=c["up"],
         V1=c["V1"], reference_batches=np.int64(doc["batches"]), reference_seconds=np.float64(doc["seconds"]))


if __name__ == "__main__":
    main(reference_dir(sys.argv))
