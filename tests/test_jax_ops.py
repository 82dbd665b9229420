"""The jax.custom_vjp adapter: importable without jax, and clear about it."""

import importlib.util

import pytest

import pyroffi_b200.jax_ops as J


@pytest.mark.skipif(importlib.util.find_spec("jax") is not None, reason="jax is installed")
def test_adapter_without_jax_raises_on_use():
    with pytest.raises(ImportError, match="needs jax"):
        J.traj_cost_vjp(object())
