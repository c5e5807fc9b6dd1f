"""Shared fixtures.  `-m gpu` tests need a B200 and the built libmsf.so;
everything else runs on the CPU (oracle, host logic, parsing, C-ABI load)."""
import hashlib
import json
import re
import shutil
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
GOLDEN = ROOT / "tests" / "golden"
sys.path.insert(0, str(ROOT / "ms-stem-fem_b200"))
sys.path.insert(0, str(ROOT / "oracle"))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200) and libmsf.so")


def golden_cases(md=False):
    """Golden cases of the ms-stem-fem driver, or (md) of ms-stem-fem-md."""
    return sorted(p.stem for p in GOLDEN.glob("*.json")
                  if bool(json.loads(p.read_text()).get("md")) == md)


def load_case(name):
    meta = json.loads((GOLDEN / (name + ".json")).read_text())
    data = dict(np.load(GOLDEN / (name + ".npz")))
    return meta, data


_SPEC_CACHE = {}


def case_dir(name, tmp_root: Path) -> Path:
    """A directory holding the case's specimen file under the name its argv
    uses; large specimens are regenerated from their seed and checked
    against the recorded sha256."""
    meta, _ = load_case(name)
    d = tmp_root / name
    d.mkdir(parents=True, exist_ok=True)
    if meta.get("md"):  # initial and replayed configurations, pre-TEM commands
        for f in (GOLDEN / name).iterdir():
            shutil.copy(f, d / f.name)
        return d
    target = d / meta["argv"][1]
    if meta["committed_specimen"]:
        shutil.copy(GOLDEN / meta["argv"][1], target)
    else:
        key = json.dumps(meta["recipe"], sort_keys=True)  # cases may share a specimen
        if key not in _SPEC_CACHE:
            sys.path.insert(0, str(GOLDEN))
            import make_golden  # the recipe that made the fixture
            gen = tmp_root / ("_gen_" + name + ".data")
            make_golden.make_specimen_file(meta["recipe"], gen)
            digest = hashlib.sha256(gen.read_bytes()).hexdigest()
            assert digest == meta["specimen_sha256"], "regenerated specimen differs"
            _SPEC_CACHE[key] = gen
        shutil.copy(_SPEC_CACHE[key], target)
    files = meta.get("files", {})
    for fname, text in files.items():  # parameter / MTF files, names made absolute
        for other in files:
            text = re.sub(r"(?<![\w./])%s(?![\w.])" % re.escape(other), str(d / other), text)
        (d / fname).write_text(text)
    return d


def case_argv(name, d):
    """The case's argv with its specimen and extra files named by absolute
    path inside the case directory `d`."""
    meta, _ = load_case(name)
    local = {meta["argv"][1]} | set(meta.get("files", {}))
    return [str(d / a) if a in local else a for a in meta["argv"]]


@pytest.fixture(scope="session")
def golden_tmp(tmp_path_factory):
    return tmp_path_factory.mktemp("golden")


def rel_err(a, b):
    a, b = np.asarray(a, float), np.asarray(b, float)
    return np.abs(a - b) / np.maximum(np.abs(b), 1e-300)


def assert_variance_close(got, ref, rtol, atol, what=""):
    """V(k) comparison: same NaN pattern, |got-ref| <= rtol*|ref| + atol.
    `atol` covers the cancellation floor of V = n*sum(A^2)/sum(A)^2 - 1,
    whose absolute resolution is ~eps of the accumulation precision."""
    got, ref = np.asarray(got, float), np.asarray(ref, float)
    assert got.shape == ref.shape, (what, got.shape, ref.shape)
    assert np.array_equal(np.isnan(got), np.isnan(ref)), (what, "NaN pattern differs")
    m = ~np.isnan(ref)
    err = np.abs(got[m] - ref[m])
    lim = rtol * np.abs(ref[m]) + atol
    bad = err > lim
    assert not bad.any(), (what, "worst", float((err / np.maximum(lim, 1e-300)).max()),
                           np.flatnonzero(m)[bad][:5], got[m][bad][:5], ref[m][bad][:5])
