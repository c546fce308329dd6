"""Shared test set-up: the ``gpu`` marker, the repository on sys.path, and golden fixtures."""
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

GOLDEN = os.path.join(ROOT, 'tests', 'golden')


def pytest_configure(config):
    config.addinivalue_line('markers', 'gpu: needs a CUDA device (B200); runs the CUDA backend through its C-ABI')


def golden(name: str, tag: str) -> dict:
    """The arrays of one fixture group, ``tag/key`` -> ``key``."""
    data = np.load(os.path.join(GOLDEN, name))
    prefix = tag + '/'
    return {key[len(prefix):]: data[key] for key in data.files if key.startswith(prefix)}


def goldenTags(name: str) -> list:
    data = np.load(os.path.join(GOLDEN, name))
    return sorted({key.split('/')[0] for key in data.files})
