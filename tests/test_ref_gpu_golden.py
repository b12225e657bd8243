"""Pins against the reference's own GPU path: outputs of gpuPairHMM (built for
sm_100a from the reference sources by oracle/Makefile) on a B200, for seeded
inputs regenerated here.  The reference keeps FP32 cells without rescue, so
its results are compared where they are finite and above -60 (normal-range
FP32); below that the reference underflows (-inf) or loses digits, and our
results are compared with the FP64 oracle instead."""
import sys
from pathlib import Path

import numpy as np
import pytest

sys.path.insert(0, str(Path(__file__).resolve().parent / "golden"))
import refgpu  # noqa: E402

import oracle  # noqa: E402
from oracle import formats  # noqa: E402
from conftest import assert_log10_close  # noqa: E402

REF_RANGE = -60.0


@pytest.mark.parametrize("name", refgpu.CASES)
def test_oracle_matches_reference_gpu(name):
    text, ref = refgpu.load(name)
    want = oracle.batch_log10(formats.to_soa(formats.parse_text(text)))
    assert len(want) == len(ref)
    ok = np.isfinite(ref) & (ref > REF_RANGE)
    assert ok.sum() > 0
    assert_log10_close(want[ok], ref[ok], what=f"oracle vs reference GPU ({name})")
    # where the reference underflowed the oracle is still finite
    assert np.all(np.isfinite(want))


@pytest.mark.gpu
@pytest.mark.parametrize("name", refgpu.CASES)
def test_engine_matches_reference_gpu(name, engine):
    import gpupairhmm_b200 as g
    text, ref = refgpu.load(name)
    recs = g.parse_records(text)
    got = engine.compute(recs.batch).astype(np.float64)
    ok = np.isfinite(ref) & (ref > REF_RANGE)
    assert_log10_close(got[ok], ref[ok], what=f"engine vs reference GPU ({name})")
    want = oracle.batch_log10(recs.batch)
    assert_log10_close(got[~ok], want[~ok], what=f"engine vs oracle where the reference underflows ({name})")
