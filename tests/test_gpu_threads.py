"""Contexts used from several host threads at once: in a fresh process four
threads each create a context and decode streams through tc_decode_j2k
concurrently, so the per-device kernel setup (attributes, occupancy) is
first reached from several threads together; every result equals a
single-threaded decode."""
import subprocess
import sys

import pytest

from conftest import ROOT

pytestmark = pytest.mark.gpu

SCRIPT = r"""
import sys, threading
import numpy as np
sys.path.insert(0, sys.argv[1])
from thousandthchicken_b200 import codec
from thousandthchicken_b200.stages import Context, Decoder
from thousandthchicken_b200.synth import gradient_noise_image
streams = [codec.encode(gradient_noise_image(384, 256, 3, 8, seed=s), 8, levels=4, reversible=s % 2 == 0,
                        mct=True, base_step=1 / 128) for s in range(4)]
results = [[None] * 4 for _ in range(4)]
errors = []
start = threading.Barrier(4)
def work(t):
    try:
        dec = Decoder(Context(0))
        start.wait()
        for k in range(4):
            results[t][k] = dec.decode(streams[(t + k) % 4])
    except Exception as e:
        errors.append(repr(e))
threads = [threading.Thread(target=work, args=(t,)) for t in range(4)]
for th in threads:
    th.start()
for th in threads:
    th.join()
assert not errors, errors
ref = [Decoder(Context(0)).decode(cs) for cs in streams]
for t in range(4):
    for k in range(4):
        assert np.array_equal(results[t][k], ref[(t + k) % 4]), (t, k)
print("ok")
"""


def test_contexts_from_threads_decode_alike():
    run = subprocess.run([sys.executable, "-c", SCRIPT, str(ROOT)], capture_output=True, text=True, timeout=600)
    assert run.returncode == 0, run.stdout[-2000:] + run.stderr[-2000:]
    assert run.stdout.strip().endswith("ok")
