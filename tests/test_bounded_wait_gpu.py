"""The bounded waits of the box-fed stencil, made to run out on purpose.

A child process sets QSB_STENCIL_COMPUTE_POLLS=1: the compute warps of
fd8_ws_kernel then give up on a ring stage after one poll of its mbarrier
(a copy that has not landed yet), leave their loop and set bit 0 of the device
error word; the producer warp, whose own waits keep the full limit, waits for
the stage releases that no longer come, runs out, waits for its copies in
flight to land and returns.  Every wait ends, the context stays usable, and
the host reads the failure from qsb_device_status.  No fault is involved."""
import json
import os
import subprocess
import sys

import pytest

pytestmark = pytest.mark.gpu
HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)

CHILD = r"""
import json, sys
import numpy as np
import torch
import qsb
import oracle as O
n, h = 32, 6.0 / 32
N = n ** 3
pos = O.bcc_positions(6.0, 1) + 0.05
tab = O.gth_tables(pos, [O.GTH_BCC] * 2, h, h, h)
H = qsb.Hamiltonian(n, n, n, h, h, h)
H.set_potential(O.seeded_potential(0, N))
H.set_projectors(*tab)
psi = torch.from_numpy(O.seeded_psi(0, 2, N)).cuda()
hp = torch.zeros_like(psi)
H.apply(psi, hp)
torch.cuda.synchronize()
word = qsb.device_status(clear=True)
after_clear = qsb.device_status()
ref = O.hamiltonian((n, n, n, h, h, h), O.seeded_potential(0, N), tab, O.seeded_psi(0, 2, N), 2)
err = float(np.linalg.norm(hp.cpu().numpy() - ref) / np.linalg.norm(ref))
x = torch.ones(1024, device="cuda") * 2.0            # the context still runs work
print(json.dumps({"word": word, "after_clear": after_clear, "err": err, "ok": float(x.sum().item())}))
"""


def test_stencil_waits_that_run_out_set_the_error_word(qsb):
    env = dict(os.environ)
    env["QSB_STENCIL_COMPUTE_POLLS"] = "1"
    env["PYTHONPATH"] = os.pathsep.join([os.path.join(ROOT, "qumasun-workshop-template_b200"),
                                         os.path.join(ROOT, "oracle"), env.get("PYTHONPATH", "")])
    r = subprocess.run([sys.executable, "-c", CHILD], env=env, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr[-2000:]
    out = json.loads(r.stdout.strip().splitlines()[-1])
    assert out["word"] & 1, out                      # a bounded wait ran out
    assert out["after_clear"] == 0, out
    assert out["err"] > 1e-6, out                    # the apply came back incomplete
    assert out["ok"] == 2048.0
    # this process (normal limits) is untouched
    assert qsb.device_status() == 0
