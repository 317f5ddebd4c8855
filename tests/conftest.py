import json
import sys
from dataclasses import fields
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))

GOLDEN = ROOT / "tests" / "golden"


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")


def params_from_json(text):
    from trench_b200.params import Params
    d = json.loads(str(text))
    names = {f.name for f in fields(Params)}
    return Params(**{k: v for k, v in d.items() if k in names})


def load_golden(name):
    with np.load(GOLDEN / name, allow_pickle=False) as d:
        out = {k: d[k] for k in d.files}
    if "params" in out:
        out["p"] = params_from_json(out.pop("params"))
    return out


@pytest.fixture(scope="session")
def golden():
    return load_golden


@pytest.fixture(scope="session")
def cuda_device():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from trench_b200 import build
    build.build()
    return 0
