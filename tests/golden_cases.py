"""Loads the golden fixtures written by tests/golden/make_golden.py."""
import json
import os

import numpy as np

from mbtrack_b200.abi import params_from_dict

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
CASES = ["single_noiseoff", "single_noise", "train_rw_hom", "feedback_hc"]


class Case:
    def __init__(self, name):
        z = np.load(os.path.join(GOLDEN, name + ".npz"), allow_pickle=False)
        self.name = name
        self.bucket = z["bucket"]
        self.np = z["np"]
        self.ib = z["ib"]
        self.Gl, self.Gv, self.Gh = z["Gl"], z["Gv"], z["Gh"]
        self.init = z["init"]
        self.init_stats = z["init_stats"]
        self.stats = z["stats"]
        self.final = z["final"]
        self.deviates = z["deviates"]
        self.vrf_phi = z["vrf_phi"]
        self.phasor = z["phasor"]
        self.params_dict = json.loads(str(z["params"]))
        self.params = params_from_dict(self.params_dict)
        self.conf = str(z["conf"])
        self.overrides = json.loads(str(z["overrides"]))
        self.turns = self.stats.shape[0]
        self.nb = len(self.bucket)

    def bunch_slices(self, flat):
        """Split a flat soa6-per-bunch buffer into [6, np] arrays."""
        out, pos = [], 0
        for n in self.np:
            out.append(flat[pos:pos + 6 * n].reshape(6, n))
            pos += 6 * n
        return out

    def conf_file(self, tmp_path):
        from tests.util import small_conf
        return small_conf(tmp_path, self.conf, **self.overrides)
