"""The JAX binding (beamax_b200.jax_ffi): imports without JAX, reports itself
unavailable and raises ImportError on use; its C++ handlers call only entry
points that include/msgb.h declares.  With JAX present (not on this machine)
the handlers would be built and registered; that path is untested here."""

import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_module_imports_and_skips_cleanly_without_jax():
    from beamax_b200 import jax_ffi

    try:
        import jax  # noqa: F401
        has_jax = True
    except ImportError:
        has_jax = False
    assert jax_ffi.available() == has_jax
    if not has_jax:
        with pytest.raises(ImportError, match="needs jax"):
            jax_ffi.register()
        with pytest.raises(ImportError, match="needs jax"):
            jax_ffi.beam_sum(None, None, None, None, None, None, None, c=1.0, L=(1.0,), periodic=(0,))


def test_ffi_handlers_call_declared_entry_points_only():
    from beamax_b200 import jax_ffi

    header = open(os.path.join(ROOT, "include", "msgb.h")).read()
    declared = set(re.findall(r"\b(msgb_[a-z0-9_]+)\s*\(", re.sub(r"/\*.*?\*/", "", header, flags=re.S)))
    src = open(jax_ffi.SRC).read()
    called = set(re.findall(r"\b(msgb_[a-z0-9_]+)\s*\(", re.sub(r"//[^\n]*", "", src)))
    assert called and called <= declared, called - declared
    for sym in jax_ffi.TARGETS.values():
        assert f"XLA_FFI_DEFINE_HANDLER_SYMBOL({sym}," in src
