"""Shared fixtures for the GPU parity tests (marked `gpu`)."""
import pytest


@pytest.fixture(scope="session")
def ctx():
    import apple_b200

    c = apple_b200.Context(0)
    info = c.device_info()
    assert info["cc"][0] == 10, info
    yield c
    c.close()
