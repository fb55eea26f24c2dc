"""Site-resolved string constraints on the device.

The reference's ``symmetry_sector_configs`` with ``string_op_diags`` /
``string_sectors`` dispatches to ``iterative_sitebased_sym_sector_configs1``
(edlgt/symmetries/symmetry_sector.py:68-145, 970-1164), which checks every
new site's state against the per-site targets (``_check_string_constraints
_on_site``, :441-476).  The device enumerator folds those checks into its
per-site allowed-state masks.  The fixtures store every input of the
reference's call and its sorted keys (tests/golden/make_golden.py string).
"""

import numpy as np
import pytest

from cases import string_case_inputs, string_case_names
from oracle import edlgt_oracle as O

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def dev():
    import torch

    assert torch.cuda.is_available(), "GPU tests need a CUDA device"
    return "cuda"


def test_string_sectors_bit_exact(golden_string, dev):
    from edgpu.symmetries import symmetry_sector_configs

    names = string_case_names(golden_string)
    assert len(names) >= 8
    for name in names:
        a = string_case_inputs(golden_string, name)
        sec = symmetry_sector_configs(**a, return_sector=True)
        ref = golden_string[f"{name}/keys"]
        keys = sec.host_keys()
        assert np.array_equal(keys, ref), name
        if len(ref) == 0:
            continue
        # the decoded table is the reference's uint16 layout
        cfg = sec.configs
        assert np.array_equal(O.keys_of(cfg, a["loc_dims"]), ref), name
        # every configuration is found at its own row
        assert np.array_equal(sec.index_of(cfg), np.arange(len(ref))), name


def test_string_sector_lookup_misses(golden_string, dev):
    """A configuration of the sector without the strings but violating them
    is not in the string sector: the lookup returns -1 for it."""
    from edgpu.symmetries import symmetry_sector_configs

    name = "su2_L12_parity"
    a = string_case_inputs(golden_string, name)
    sec = symmetry_sector_configs(**a, return_sector=True)
    base = dict(a)
    base.pop("string_op_diags")
    base.pop("string_sectors")
    full = symmetry_sector_configs(**base, return_sector=True)
    assert len(full) == int(golden_string[f"{name}/base_dim"])
    idx = sec.index_of(full.configs)
    inside = np.isin(full.host_keys(), golden_string[f"{name}/keys"])
    assert np.all(idx[~inside] == -1)
    assert np.array_equal(np.sort(idx[inside]), np.arange(len(sec)))
