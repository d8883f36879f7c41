"""The drop-in (``plugin.install``) against the reference package itself, on the CPU.

These tests import the reference from its checkout (``CDFT_REFERENCE``, default the build
container's read-only tree) and are skipped where it is absent: the reference does not travel to
the GPU box. They check that ``install`` rebinds exactly the seams the reference's CUDA path
dispatches through, that ``uninstall`` restores them, that the CPU audit path stays bit-for-bit the
reference's with the plugin installed, and the ``CDFT_NATIVE`` switch.
"""

from __future__ import annotations

import dataclasses
import importlib
import os
import sys
from pathlib import Path

import pytest

REFERENCE = Path(os.environ.get("CDFT_REFERENCE", "/root/reference"))


@pytest.fixture(scope="module")
def cdft():
    if not (REFERENCE / "src" / "cdft").is_dir():
        pytest.skip("the reference checkout is not available here")
    os.environ.setdefault("PYTHONDONTWRITEBYTECODE", "1")
    sys.dont_write_bytecode = True
    for p in (str(REFERENCE / "src"), str(REFERENCE)):
        if p not in sys.path:
            sys.path.insert(0, p)
    return importlib.import_module("cdft")


@pytest.fixture()
def plugin(pkg):
    mod = importlib.import_module("cdft_b200.plugin")
    yield mod
    mod.uninstall()


def test_mode_switch(pkg, monkeypatch):
    plugin = importlib.import_module("cdft_b200.plugin")
    assert plugin.requested_mode("") == "auto"
    assert plugin.requested_mode(" ON ") == "on"
    assert plugin.requested_mode("off") == "off"
    with pytest.raises(ValueError, match="CDFT_NATIVE"):
        plugin.requested_mode("yes")
    monkeypatch.setenv("CDFT_NATIVE", "autoo")
    with pytest.raises(ValueError, match="autoo"):
        plugin.install()
    assert not plugin.installed()


def _seam_values(plugin):
    out = {}
    for module, path, _ in plugin.SEAMS:
        owner, name = plugin._owner(module, path)
        out[(module, path)] = owner.__dict__[name] if isinstance(owner, type) else getattr(owner, name)
    return out


def test_install_binds_exactly_the_seams_and_uninstall_restores(cdft, plugin):
    before = _seam_values(plugin)
    rec = plugin.install("auto")
    assert rec["tier"] == "native-sm100a" and rec["mode"] == "auto"
    after = _seam_values(plugin)
    for module, path, replacement in plugin.SEAMS:
        assert after[(module, path)] is replacement, (module, path)
        assert before[(module, path)] is not replacement
    # the names the reference's drivers import by name were rebound in their own modules
    import cdft.scf.loop as loop
    import cdft.scf.noninteracting as nonint
    assert loop.graphed_filter_for is plugin.graphed_filter_for
    assert nonint.graphed_filter_for is plugin.graphed_filter_for
    assert plugin.install("auto")["seams"] == rec["seams"]  # idempotent
    plugin.uninstall()
    assert _seam_values(plugin) == before


def test_off_binds_nothing(cdft, plugin):
    before = _seam_values(plugin)
    rec = plugin.install("off")
    assert rec["tier"] == "reference" and rec["seams"] == []
    assert _seam_values(plugin) == before


def test_cpu_audit_path_is_unchanged(cdft, plugin):
    """A CPU solve of the reference with the plugin installed is bit for bit the one without: every
    replacement hands CPU tensors to the reference's own code."""
    from contract import MixingConfig, MixingScheme
    from cdft.config import ALL_ELECTRON_NUMERICS
    from cdft.physics_config import helium, lda_functional
    from cdft.scf.solve import solve_scenario

    base = ALL_ELECTRON_NUMERICS
    num = dataclasses.replace(
        base, grid=dataclasses.replace(base.grid, spacing=0.5, box_lengths=(8.0, 8.0, 8.0)),
        eigen=dataclasses.replace(base.eigen, cross_check=False),
        mixing=MixingConfig(scheme=MixingScheme.LINEAR, alpha=0.3))
    scenario = dataclasses.replace(helium(), xc=lda_functional("vwn"))

    def solve():
        art = solve_scenario(scenario, num, derive_grid=False)
        assert art.result is not None, art.error_message
        return art.result.energies, art.result.eigenvalues, art.result.n_iterations

    want = solve()
    plugin.install("on")  # forced: still no CPU call may go native
    got = solve()
    rec = plugin.record()
    assert got[0] == want[0] and got[2] == want[2]
    assert got[1].tolist() == want[1].tolist()
    assert rec["native_calls"] == {} and rec["reference_calls"] == {}
