import importlib.util
import pathlib
import sys

ROOT = pathlib.Path(__file__).resolve().parent.parent
for p in (str(ROOT), str(ROOT / "tests")):
    if p not in sys.path:
        sys.path.insert(0, p)

# The package directory is named oxideav-h266_b200 (not an identifier); register
# it under the importable name oxideav_h266_b200.
if "oxideav_h266_b200" not in sys.modules:
    _pkg = ROOT / "oxideav-h266_b200"
    _spec = importlib.util.spec_from_file_location("oxideav_h266_b200", _pkg / "__init__.py",
                                                   submodule_search_locations=[str(_pkg)])
    _mod = importlib.util.module_from_spec(_spec)
    sys.modules["oxideav_h266_b200"] = _mod
    _spec.loader.exec_module(_mod)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); run with -m gpu")
