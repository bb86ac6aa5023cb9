"""``.grim`` export against the reference's own archives (``tests/golden/grim``, made by
``tests/golden/make_grim_golden.py`` with the reference's ``export_result_to_grim``):
every stored array and string equal, for format versions 1 and 2, single-polarisation,
co-polarised and raw-amplitude-free results."""
import importlib.util
import os

import numpy as np
import pytest

from grim_20261007_b200 import grimfile
from tests.conftest import GOLDEN

GRIM_DIR = os.path.join(GOLDEN, 'grim')


def _cases():
    spec = importlib.util.spec_from_file_location('make_grim_golden', os.path.join(GOLDEN, 'make_grim_golden.py'))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod.results()


CASES = _cases()


def _load(path):
    with np.load(path, allow_pickle=False) as z:
        return {k: z[k] for k in z.files}


@pytest.mark.parametrize('version', [1, 2])
@pytest.mark.parametrize('name', sorted(CASES))
def test_export_equals_the_reference_archive(tmp_path, name, version):
    res, kw = CASES[name]
    out = grimfile.export_result_to_grim(res, str(tmp_path / name), format_version=version, **kw)
    assert len(out) == 1 and out[0].endswith('.grim') and os.path.isabs(out[0])
    got = _load(out[0])
    ref = _load(os.path.join(GRIM_DIR, f'{name}_v{version}.grim'))
    assert set(got) == set(ref)
    for key in ref:
        assert got[key].dtype == ref[key].dtype, key
        assert got[key].shape == ref[key].shape, key
        if got[key].dtype.kind in 'fc':
            np.testing.assert_array_equal(got[key], ref[key], err_msg=key)
        else:
            assert np.array_equal(got[key], ref[key]), key


@pytest.mark.parametrize('name', ['tm', 'co'])
def test_version_two_reads_back_as_the_version_one_keys(tmp_path, name):
    res, kw = CASES[name]
    v2 = grimfile.export_result_to_grim(res, str(tmp_path / 'a.grim'), format_version=2, **kw)[0]
    v1 = _load(os.path.join(GRIM_DIR, f'{name}_v1.grim'))
    back = grimfile.load_grim_npz(v2)
    for key in ('rcs_power', 'rcs_phase', 'rcs_amp_real', 'rcs_amp_imag', 'azimuths', 'frequencies', 'polarizations'):
        assert back[key].shape == v1[key].shape, key
    np.testing.assert_array_equal(back['rcs_amp_real'], v1['rcs_amp_real'])
    np.testing.assert_array_equal(back['rcs_amp_imag'], v1['rcs_amp_imag'])
    np.testing.assert_array_equal(back['rcs_phase'], v1['rcs_phase'])
    np.testing.assert_allclose(back['rcs_power'], v1['rcs_power'], rtol=2e-7)


def test_invalid_results_are_refused_with_the_reference_messages(tmp_path):
    res, kw = CASES['tm']
    bad = dict(res, samples=[dict(r) for r in res['samples']])
    bad['samples'][2]['rcs_linear'] *= 1.01
    with pytest.raises(ValueError, match='Invalid solver sample at index 2: rcs_linear .* is inconsistent'):
        grimfile.export_result_to_grim(bad, str(tmp_path / 'x'))
    bad = dict(res, samples=res['samples'][:-3])
    with pytest.raises(ValueError, match='complete rectangular'):
        grimfile.export_result_to_grim(bad, str(tmp_path / 'x'))
    dup = dict(res, samples=[dict(r) for r in res['samples']] + [dict(res['samples'][0])])
    with pytest.raises(ValueError, match='Duplicate sample conflict'):
        grimfile.export_result_to_grim(dup, str(tmp_path / 'x'))
    with pytest.raises(ValueError, match='single-channel fallback was refused'):
        grimfile.export_result_to_grim(dict(res, polarizations=['VV']), str(tmp_path / 'x'))
    with pytest.raises(ValueError, match='format_version must be 1 or 2'):
        grimfile.export_result_to_grim(res, str(tmp_path / 'x'), format_version=3)
    assert not any(p.name.startswith('.') for p in tmp_path.iterdir())  # no temporary file left behind
