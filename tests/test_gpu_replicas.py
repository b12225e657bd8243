"""Replicas on the GPU: replicas.run with one engine per listed device gives
the single engine's scores bitwise (a pair's result depends only on its own
read and haplotype).  Only one GPU is available here, so the replicas share
it; on a node with several GPUs the same call takes their ordinals."""
import numpy as np
import pytest

import gpupairhmm_b200 as g
from gpupairhmm_b200 import replicas, synth

pytestmark = pytest.mark.gpu


def test_replicas_match_one_engine(engine):
    b = synth.concat([synth.config1(seed=61, regions=60), synth.config2(seed=62, regions=2),
                      synth.config3(seed=63, regions=1)])
    want = engine.compute(b)
    for devices in ([0], [0, 0], [0, 0, 0]):
        np.testing.assert_array_equal(replicas.run(b, devices=devices), want)
