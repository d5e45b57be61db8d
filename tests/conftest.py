import os
import sys

# OpenCV reads OpenEXR files (the image decoders' reference) only when asked.
os.environ.setdefault('OPENCV_IO_ENABLE_OPENEXR', '1')

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line('markers', 'gpu: needs a CUDA GPU (B200, sm_100a)')


def _load_build_module():
    import importlib.util
    spec = importlib.util.spec_from_file_location('vision_b200_build', os.path.join(ROOT, 'vision_b200', 'build.py'))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def _ensure_built():
    vb_build = _load_build_module()
    if not vb_build.up_to_date():
        # nvcc cross-compiles sm_100a without a GPU; on a box without nvcc the
        # prebuilt library that travelled with the repository is used.
        try:
            vb_build.build()
        except Exception as e:  # pragma: no cover - reported by the import below
            print('library build failed: %s' % e)
    import oracle
    oracle.build()


_ensure_built()


@pytest.fixture(scope='session')
def vb():
    import vision_b200
    return vision_b200


@pytest.fixture(scope='session')
def gpu_ctx(vb):
    import torch
    if not torch.cuda.is_available():
        pytest.skip('no CUDA device')
    return vb.Context(0)


@pytest.fixture(scope='session')
def host_ctx(vb):
    return vb.Context(-1)
