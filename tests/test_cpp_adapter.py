"""GPU: the C++ adapter (BuildCuda32/64, BuildCudaStorage) through its test
driver, against the reference's divsufsort64 build."""
import subprocess
from pathlib import Path

import numpy as np
import pytest

import oracle
from sufkit_b200 import build as sgbuild
from sufkit_b200 import synth

pytestmark = pytest.mark.gpu


def load(path):
    return np.fromfile(path, dtype=np.uint64)


def test_cpp_adapter_matches_reference(tmp_path):
    driver = sgbuild.build_driver()
    text = synth.repeat_rich_100mbp(scale=0.01).logical_text()
    (tmp_path / "t.bin").write_bytes(text.tobytes())
    run = subprocess.run([str(driver), str(tmp_path / "t.bin"), str(tmp_path / "o")],
                         capture_output=True, text=True, timeout=300)
    assert run.returncode == 0, run.stdout + run.stderr
    if oracle.ref() is not None:
        sa, isa, lcp, _ = oracle.ref_adapter(text, 64)
    else:
        sa, isa, lcp = oracle.full_build(text)
    assert (load(tmp_path / "o.sa64") == sa).all()
    assert (load(tmp_path / "o.isa64") == isa).all()
    assert (load(tmp_path / "o.lcp64") == lcp).all()
    assert (load(tmp_path / "o.sa32") == sa).all()
    assert (load(tmp_path / "o.lcp32") == lcp).all()
    _, low, high = oracle.pack(sa, text.size, 40)
    assert (load(tmp_path / "o.sa40low") == low).all()
    assert (load(tmp_path / "o.sa40high") == high).all()
    primary, pos, val = oracle.bytecode(text, sa, isa, 32)
    assert (load(tmp_path / "o.primary") == primary).all()
    assert (load(tmp_path / "o.anchor_pos") == pos).all()
    assert (load(tmp_path / "o.anchor_val") == val).all()
    if oracle.ref() is not None:
        sa_k, isa_k, lcp_k = oracle.ref_adapter_sampled(text, 4, 64)
    else:
        sa_k, isa_k, lcp_k = oracle.sample(sa, lcp, 4)
    assert (load(tmp_path / "o.sa_k4") == sa_k).all()
    assert (load(tmp_path / "o.isa_k4") == isa_k).all()
    assert (load(tmp_path / "o.lcp_k4") == lcp_k).all()
