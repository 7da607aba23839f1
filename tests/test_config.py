"""The product's C++ condition parser against the oracle's restatement of
src/Init.mm on the reference's own condition files (no GPU needed)."""
import glob
import json
import os

import pytest

from gample_b200 import capi
from oracle import config as ocfg
from tests.helpers import GOLDEN, condition

CONDITIONS = sorted(glob.glob(os.path.join(GOLDEN, "*.json")))


def _cmp(a, b, path=""):
    if isinstance(b, dict):
        for k, v in b.items():
            if k in a:
                _cmp(a[k], v, path + "." + k)
    elif isinstance(b, list):
        assert len(a) == len(b), path
        for i, (x, y) in enumerate(zip(a, b)):
            _cmp(x, y, f"{path}[{i}]")
    else:
        assert a == b, (path, a, b)


@pytest.mark.parametrize("path", CONDITIONS, ids=[os.path.basename(p) for p in CONDITIONS])
def test_parser_matches_reference_semantics(path):
    try:
        expect = ocfg.parse(path)
    except ocfg.ConfigError:
        with pytest.raises(capi.GampleError) as ei:
            capi.Init(path)
        assert ei.value.status == 2
        return
    got = capi.Init(path).dump()
    _cmp(got, expect)


def test_defaults_and_derived_values():
    c = condition(ngx=10, ngy=20, order=5, ppc=3)
    del c["ParamForField"]["BorisOrder"]
    got = capi.Init(c).dump()
    assert got["field"]["ngb"] == 2 and got["field"]["BorisOrder"] == 2
    assert got["particles"][0]["pNum"] == 600
    # w = n dx dy / ppc (src/Init.mm:194-196)
    assert abs(got["particles"][0]["w"] - 5e10 * 0.005 * 0.005 / 3) < 1e-6
    # ToleranceForPoisson is a float member (src/Init.h:35)
    import struct
    assert got["comp"]["tolerance"] == struct.unpack("f", struct.pack("f", 1e-8))[0]


@pytest.mark.parametrize("mutate,section", [
    (lambda c: c.pop("FlagForEquation"), "FlagForEquation"),
    (lambda c: c["ParamForParticle"][0].update(pNumSetMethod="bogus"), "pNumSet"),
    (lambda c: c["ParamForParticle"][0].update(WeightSetMethod="bogus"), "WeightSet"),
    (lambda c: c.update(SourceForParticle=[{"SrcSetMethod": "bogus"}]), "SrcSet"),
    (lambda c: c.update(BoundaryConditionForField={}), "BoundaryConditionForField"),
])
def test_rejections_match_reference(mutate, section):
    c = condition()
    mutate(c)
    with pytest.raises(ocfg.ConfigError):
        ocfg.parse(c)
    with pytest.raises(capi.GampleError) as ei:
        capi.Init(c)
    assert ei.value.status == 2


def test_malformed_json_is_a_config_error():
    with pytest.raises(capi.GampleError) as ei:
        capi.Init("{\"FlagForEquation\": {")
    assert ei.value.status == 2
    with pytest.raises(capi.GampleError):
        capi.Init(os.path.join(GOLDEN, "does_not_exist.json"))


def test_build_addition_keys_are_ignored_by_reference_schema():
    c = condition(deposit_mode=1)
    expect = ocfg.parse(c)   # the reference's parser ignores unknown keys
    got = capi.Init(c).dump()
    _cmp(got, expect)
    assert json.dumps(got)
