"""The full-size workloads still produce the inputs the reference digests were made from.

tests/golden/fullsize.json records, beside the digests of the reference's outputs,
the digests of the inputs rockseis_b200.workloads generated for them.  If a
generator changes, the GPU full-size parity tests would compare against outputs of
different inputs; this CPU test catches that first.
"""
import json
import os

import numpy as np

from rockseis_b200 import workloads as W

GOLD = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "fullsize.json")))


def test_workload_inputs_unchanged():
    for name, arrays in (("c1", W.acoustic2d_c1()), ("c2", W.elastic2d_c2()), ("c3", W.fwi_c3())):
        for k, a in enumerate(arrays):
            assert W.digest(np.asarray(a)) == GOLD["inputs"][f"{name}_input{k}"], (name, k)


def test_golden_samples_match_digest_records():
    s = np.load(os.path.join(os.path.dirname(__file__), "golden", "fullsize.npz"))
    for k in s.files:
        g = GOLD[k]
        full = g["shape"]
        assert s[k].dtype == np.dtype(g["dtype"]), k
        # every kept sample is a strided view of the full array, so it cannot exceed its extreme
        assert np.abs(s[k]).max() <= g["absmax"], k
        assert all(a <= b for a, b in zip(s[k].shape, full)), k
