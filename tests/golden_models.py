"""Loads the committed 1AZP golden fixture (tests/golden/1azp_models.npz)."""
import os

import numpy as np

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def azp(family):
    """Receptor / ligand parameter dicts of 1AZP typed for `family`."""
    d = np.load(os.path.join(GOLDEN, "1azp_models.npz"))
    tab = "dna" if family == "dna" else "pydock"

    def side(s):
        m = dict(coords=d[f"{tab}_{s}_coords"], ele=d[f"{tab}_{s}_ele"],
                 vdw=d[f"{tab}_{s}_vdw"], radius=d[f"{tab}_{s}_radius"])
        if family == "dna":
            m["heavy"] = d[f"dna_{s}_heavy"]
        m["is_h"] = d[f"{s}_is_h"]
        return m

    return side("rec"), side("lig")
