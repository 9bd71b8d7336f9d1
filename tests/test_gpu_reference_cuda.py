"""The reference's own CUDA kernels (built for sm_100a from its sources by
oracle/build_ref_cuda.sh) against this library, on the same inputs.

The reference engine's HMult -> relinearize -> rescale operator sequence
runs on CUDA tensors through the reference's CUDA kernels, with its default
CUDA NTT policy, at slots32768_scale40_levels34_int64 (levels 0 and 30).
The fused path of this library, with the key switch's basis conversions on
the CUDA cores and on the int8 tensor cores, must be integer-equal to it on
every ciphertext, except where the reference's CUDA result also differs
from the reference's own CPU kernels: there it must equal the CPU kernels'
result.  (On B200 the reference's CUDA path was seen to differ from its CPU
kernels in single words of a few ciphertexts of a batch of 32.)  The run is
a child process: the reference's library defines the same operator schemas
as the CPU-only reference library that other tests load."""

import json
import os
import subprocess
import sys

import pytest

from oracle.ref_pipeline import available

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.mark.skipif(not available("cuda"), reason="oracle/_ref/libfhelium_ref_ops_cuda.so not built")
@pytest.mark.parametrize("level,batch", [(0, 3), (30, 2), (0, 12)])
def test_reference_cuda_kernels_equal_ours(level, batch):
    cmd = [sys.executable, "-m", "oracle.ref_cuda", "--batch", str(batch), "--steps", "1", "--level", str(level),
           "--arbiter", str(batch)]
    res = subprocess.run(cmd, cwd=ROOT, capture_output=True, text=True, timeout=900)
    assert res.returncode == 0, res.stderr[-3000:]
    line = json.loads(res.stdout.strip().splitlines()[-1])
    assert line["forms_bit_identical"] is True
    # where the reference's CUDA kernels differ (single words, seen at larger
    # batches), its CPU kernels must side with this library
    bad = line["mismatching_ciphertexts"]
    verdicts = line.get("arbitrated", {})
    assert len(bad) == len(verdicts), "every mismatch arbitrated"
    for i, v in verdicts.items():
        assert v["reference_cpu_equals_ours"] and not v["reference_cpu_equals_reference_cuda"], (i, v)
