"""Argument checks of the differentiable trajectory that run before any kernel call."""
import pytest
import torch


def test_trajectory_rejects_negative_segment_length():
    from openonda_b200 import autodiff

    x = torch.zeros((4, 3), dtype=torch.float64)
    s = torch.ones(4, dtype=torch.float64)
    with pytest.raises(ValueError, match="checkpoint_every"):
        autodiff.trajectory(x, x, s, None, 0.01, 3, "fp64", checkpoint_every=-1)
    with pytest.raises(ValueError, match="steps"):
        autodiff.trajectory(x, x, s, None, 0.01, -2, "fp64", checkpoint_every=2)


def test_trajectory_of_zero_steps_returns_the_initial_state():
    from openonda_b200 import autodiff

    x = torch.zeros((4, 3), dtype=torch.float64)
    s = torch.ones(4, dtype=torch.float64)
    for every in (0, None, 5):
        xT, aT = autodiff.trajectory(x, x, s, None, 0.01, 0, "fp64", checkpoint_every=every)
        assert xT is x and aT is x
