"""GPU parity of the engine's schedule switches: the fused two-layer
schedule (FQ_FUSE=1, the default) or one sweep per pass (FQ_FUSE=0), with
and without the L2 prefetch of the phase pass (FQ_PREFETCH).
The mode is read once per process, so each runs in a child process; states and <C> are checked against the oracle."""
import json
import os
import subprocess
import sys

import numpy as np
import pytest

from conftest import ROOT, PKG, ENERGY_RTOL, assert_state_close, complete_int, gnp_fp, angles

pytestmark = pytest.mark.gpu

CHILD = r"""
import json, sys
import numpy as np
sys.path.insert(0, %(pkg)r)
import forqaoa
cases = json.loads(sys.stdin.read())
out = []
with forqaoa.Context(0) as ctx:
    for c in cases:
        W = np.array(c["W"]); g = np.array(c["g"]); b = np.array(c["b"])
        st = ctx.state(c["n"])
        e = ctx.qaoa_forward(st, W, g, b)
        psi = st.to_host()
        st.free()
        out.append({"e": e, "re": psi.real.tolist(), "im": psi.imag.tolist()})
print(json.dumps(out))
"""


def cases():
    rng = np.random.default_rng(77)
    out = []
    for n, kind, P in ((13, "int", 2), (16, "fp", 3), (18, "int", 2), (20, "int", 3),
                       (21, "fp", 1), (17, "neg", 2), (21, "int", 4), (19, "fp", 3)):
        W = {"int": complete_int(n, rng), "fp": gnp_fp(n, rng),
             "neg": complete_int(n, rng, -6, 6)}[kind]
        g, b = angles(rng, P)
        out.append({"n": n, "W": W.tolist(), "g": g.tolist(), "b": b.tolist()})
    return out


@pytest.mark.parametrize("prefetch,fuse", [("1", "1"), ("0", "1"), ("1", "0"), ("0", "0")])
def test_pass_modes_match_oracle(oracle, prefetch, fuse):
    cs = cases()
    env = dict(os.environ, FQ_PREFETCH=prefetch, FQ_FUSE=fuse)
    res = subprocess.run([sys.executable, "-c", CHILD % {"pkg": PKG}], input=json.dumps(cs),
                         capture_output=True, text=True, env=env, timeout=600)
    assert res.returncode == 0, res.stderr[-2000:]
    got = json.loads(res.stdout.strip().splitlines()[-1])
    for c, r in zip(cs, got):
        W, g, b = np.array(c["W"]), np.array(c["g"]), np.array(c["b"])
        want = oracle.qaoa_logical(W, g, b)
        psi = np.array(r["re"]) + 1j * np.array(r["im"])
        assert_state_close(psi, want, what=f"N={c['n']} FQ_FUSE={fuse} FQ_PREFETCH={prefetch}")
        eo = oracle.expectation(want, W)
        assert abs(r["e"] - eo) <= ENERGY_RTOL * max(1.0, abs(eo))
