"""The shipped learned-preconditioner weights: the compiled-in table
(cfdapp_b200/csrc/mg_trained.inc) is the training record
(cfdapp_b200/mg_weights.json), checksummed, point-symmetric and finite."""
import hashlib
import json
import os
import re

import numpy as np

PKG = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "cfdapp_b200")


def _load():
    with open(os.path.join(PKG, "mg_weights.json")) as f:
        return json.load(f)


def test_json_checksum_and_shape():
    d = _load()
    sets = d["sets"]
    blob = json.dumps({k: {kk: vv for kk, vv in v.items() if kk != "record"} for k, v in sets.items()},
                      sort_keys=True).encode()
    assert hashlib.sha256(blob).hexdigest() == d["sha256"]
    for dim, v in sets.items():
        k = np.array(v["kernels"], dtype=np.float32)
        assert k.shape == (v["levels"], 27)
        assert np.all(np.isfinite(k)) and np.all(np.isfinite(v["coarse_weights"]))
        assert np.array_equal(k, k[:, ::-1])  # point-symmetric
        if dim == "2":
            assert not np.any(k[:, :9]) and not np.any(k[:, 18:])
        rec = v["record"]
        assert sum(rec["trained_validation_iterations"]) < sum(rec["untrained_validation_iterations"])


def test_compiled_table_matches_the_record():
    d = _load()
    text = open(os.path.join(PKG, "csrc", "mg_trained.inc")).read()
    assert d["sha256"] in text
    for dim, v in d["sets"].items():
        block = text[text.index(f"if (dim == {dim})"):]
        rows = re.findall(r"\{([^{}]*)\},", block.split("};")[0])
        k = np.array([[float(x.rstrip("f")) for x in r.split(",")] for r in rows], dtype=np.float32)
        assert np.array_equal(k, np.array(v["kernels"], dtype=np.float32))
