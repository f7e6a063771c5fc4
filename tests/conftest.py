import os
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(ROOT / 'oracle'))

# the reference tree (read only by the oracle pin tests); LSS_REFERENCE_ROOT overrides it
REFERENCE = Path(os.environ.get('LSS_REFERENCE_ROOT', '/root/reference'))
KS_SITE = REFERENCE / 'src/Python/run_online_spikes/Lib/site-packages'
GOLDEN = Path(__file__).resolve().parent / 'golden'


def pytest_configure(config):
    config.addinivalue_line('markers', 'gpu: needs a CUDA device (B200)')


@pytest.fixture(scope='session')
def reference_ks():
    """The vendored Kilosort4 modules of the reference, when the tree exists."""
    if not KS_SITE.exists():
        pytest.skip('reference tree not present')
    import types
    import warnings
    warnings.filterwarnings('ignore')
    sys.path.insert(0, str(KS_SITE))
    sys.modules.setdefault('faiss', types.ModuleType('faiss'))
    from kilosort import template_matching, preprocessing, io as ksio
    return types.SimpleNamespace(tm=template_matching, pp=preprocessing, io=ksio)
