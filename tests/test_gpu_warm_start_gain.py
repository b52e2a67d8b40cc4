"""What the trained warm-start networks gain over the solver without them — needs a B200.

Each packaged model is run on held-out scenes of its family against the plain solver (the reference's uniform
initial guess) and against the same guess without the network (p*/m and the previous step's correction); all
three solve to the same relative residual.  The gains asserted are the CR iterations per step measured on these
seeds; wall time is not asserted (the network's inference costs more than the iterations it saves: see the
training report in the profiles).
"""
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.join(os.path.dirname(HERE), "mpmsnow_b200")


def _net(name):
    from mpmsnow_b200 import build
    from mpmsnow_b200.learned import WarmStartNet
    build.build()
    net = WarmStartNet(seed=0)
    net.load_state_dict(dict(np.load(os.path.join(PKG, name))))
    return net


def test_slab_model_reduces_cr_iterations():
    """The slab model on the four held-out slab sections, 60 steps each: fewer CR iterations than plain CR by a
    wide margin (the p*/m + history guess), and fewer than the same guess without the network, on the mean over
    the seeds (measured 7.20 against 7.30, every seed lower)."""
    from mpmsnow_b200 import warm_start_train as T
    net = _net("warm_start_slab.npz")
    rows = T.compare_in_step("slab", [4000, 4001, 4002, 4003], net, steps=60)
    plain = np.mean([r["plain"]["iterations_per_step"] for r in rows])
    learned = np.mean([r["learned"]["iterations_per_step"] for r in rows])
    base = np.mean([r["base_only"]["iterations_per_step"] for r in rows])
    for r in rows:
        print(f"seed {r['seed']}: plain {r['plain']['iterations_per_step']:.2f}, learned "
              f"{r['learned']['iterations_per_step']:.2f}, without the network {r['base_only']['iterations_per_step']:.2f}")
    print(f"slab sections: CR iterations per step plain {plain:.2f}, learned {learned:.2f}, without the network "
          f"{base:.2f}")
    assert learned < 0.7 * plain
    assert learned < base


def test_snowball_model_reduces_cr_iterations():
    from mpmsnow_b200 import warm_start_train as T
    net = _net("warm_start_snowball.npz")
    rows = T.compare_in_step("snowball", [2000, 2001, 2004], net, steps=40)
    plain = np.mean([r["plain"]["iterations_per_step"] for r in rows])
    learned = np.mean([r["learned"]["iterations_per_step"] for r in rows])
    base = np.mean([r["base_only"]["iterations_per_step"] for r in rows])
    print(f"snowball drops: CR iterations per step plain {plain:.2f}, learned {learned:.2f}, p*/m alone {base:.2f}")
    assert learned < 0.85 * plain      # measured over 40 steps on all 20 held-out seeds: 12.1 vs 16.4
