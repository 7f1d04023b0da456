"""A request built by the library's host pipeline from input.yaml text
(sdft_input_from_yaml) solves on the device to the state of the request the
Python host builds from the same text."""
import copy

import numpy as np
import pytest
import yaml

from softdft_b200 import native, workloads
from softdft_b200.api import setup_request
from softdft_b200.host.descriptor import numerics_from_dict
from tests.helpers import rel

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("np_", [256, 243])
def test_yaml_request_solves_like_the_python_request(np_):
    ds = workloads.weak_acid_slit(np_, 0.05, 8, 4.5, 7.0, 0.1, 0.3)
    ds["numerical"] = dict(ds["numerical"], tole=1e-10, max_iters=8000)
    text = yaml.safe_dump(ds, sort_keys=False)
    inp = native.Input(text)
    dev_c = native.DeviceSystem(inp.descriptor())
    dev_p = native.DeviceSystem(setup_request(copy.deepcopy(ds)).descriptor)
    num = inp.numerics()
    it_c, err_c, rc_c = dev_c.solve(num)
    it_p, err_p, rc_p = dev_p.solve(numerics_from_dict(ds["numerical"]))
    assert rc_c == 0 and rc_p == 0
    assert rel(dev_c.get_x(), dev_p.get_x()) < 1e-7
    _, b_c, _ = dev_c.densities()
    _, b_p, _ = dev_p.densities()
    assert rel(b_c, b_p) < 1e-7
