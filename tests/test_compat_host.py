"""The drop-in aliasing of the reference's module paths (no GPU): scripts
written against ``janus.*`` import janus_b200's modules."""
import sys
import types

import pytest

from janus_b200 import compat


@pytest.fixture
def clean_modules(monkeypatch):
    for name in list(compat._MODULES):
        monkeypatch.delitem(sys.modules, name, raising=False)
    yield
    for name in list(compat._MODULES):
        sys.modules.pop(name, None)


def test_reference_paths_resolve_to_janus_b200(clean_modules):
    compat.install_as_janus()
    import janus.green
    import janus.material.elastic.linear.isotropic as material
    import janus.operators

    import janus_b200.green
    import janus_b200.operators
    assert janus.green is janus_b200.green
    assert janus.operators is janus_b200.operators
    mat = material.create(1.0, 0.3, 2)
    assert mat.dim == 2 and abs(mat.k - 1.0 / (1.0 - 2 * 0.3)) < 1e-15


def test_a_foreign_janus_package_is_not_replaced(clean_modules, monkeypatch):
    foreign = types.ModuleType("janus")
    foreign.__file__ = "/elsewhere/janus/__init__.py"
    monkeypatch.setitem(sys.modules, "janus", foreign)
    with pytest.raises(RuntimeError):
        compat.install_as_janus()
    compat.install_as_janus(force=True)
    assert sys.modules["janus"].__name__ == "janus_b200"
