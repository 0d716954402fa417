"""Host seeds equal the reference's CPU seeds element for element."""
import numpy as np

from becgpp_b200.config import default_cfg
from becgpp_b200.grid import make_grid
from becgpp_b200.seeds import make_seed


def test_seeds_match_reference(golden):
    arr, meta = golden("seeds")
    for name, kw in meta.items():
        c = default_cfg(mode="single", **kw)
        G = make_grid(c)
        s = make_seed(G, c, device="cpu").numpy()
        ref = arr[name]
        err = np.max(np.abs(s - ref)) / np.max(np.abs(ref))
        assert err < 1e-14, (name, err)
