"""ParticleSystem host-side behaviour that needs no GPU: constructor validation with the
reference's messages (vpmModule.py:117-184) and the LES/BDF constants."""
import numpy as np
import pytest

from openonda_b200.vpm import vpmModule as v


def test_constructor_validation_messages():
    with pytest.raises(TypeError, match="time_step_size must be a float or int"):
        v.ParticleSystem(time_step_size="0.1")
    with pytest.raises(ValueError, match="Invalid time integration method 'RK5'"):
        v.ParticleSystem(time_integration_method="RK5")
    with pytest.raises(ValueError, match="Invalid viscous scheme"):
        v.ParticleSystem(viscous_scheme="Spectral")
    with pytest.raises(ValueError, match="'viscous_scheme' must be None"):
        v.ParticleSystem(flow_model="Potential", viscous_scheme="PSE")
    with pytest.raises(ValueError, match="must be 'CoreSpreading' or 'PSE'"):
        v.ParticleSystem(flow_model="LES", viscous_scheme=None)
    with pytest.raises(ValueError, match="Invalid processing unit 'CPU'"):
        v.ParticleSystem(processing_unit="CPU")
    with pytest.raises(ValueError, match="unknown precision"):
        v.ParticleSystem(precision="fp16")
    with pytest.raises(ValueError, match="Invalid LES coefficient scheme"):
        v.ParticleSystem(flow_model="LES", viscous_scheme="PSE", les_coefficient="germano")
    assert v.ParticleSystem().les_coefficient == "reference"


def test_defaults_follow_the_reference():
    ps = v.ParticleSystem(flow_model="LES", viscous_scheme="CoreSpreading")
    assert ps.Cnu == pytest.approx(0.02958)
    assert ps.monitor_variables == ["Circulation", "Linear Impulse", "Angular Impulse",
                                    "Kinetic Energy", "Enstrophy", "Helicity"]
    assert ps.flow_model_description == "(ω.∇)u + (ν+νt)(∇²)ω"
    assert len(ps) == 0


def test_highest_nonzero_indices():
    import numpy as np

    a = np.array([0.0, 3.0, 1.0, 0.0, 2.0])
    assert list(v.get_highest_nonzero_indices(a, top_percentage=50)) == [1]
    assert list(v.get_highest_nonzero_indices(a, strength_threshold=1.5)) == [1, 4]


def test_get_highest_nonzero_indices_matches_reference():
    """vpmModule.get_highest_nonzero_indices (vpmModule.py:1124-1166) on the reference's own
    output (tests/golden/manage.npz)."""
    from conftest import golden
    from openonda_b200.vpm.vpmModule import get_highest_nonzero_indices

    g = golden("manage.npz")
    mags = g["highest/mags"]
    assert np.array_equal(get_highest_nonzero_indices(mags, top_percentage=10), g["highest/top10"])
    thr = float(np.percentile(mags, 80))
    assert np.array_equal(get_highest_nonzero_indices(mags, strength_threshold=thr),
                          g["highest/above"])
