"""Test-side name for the package's quotient-rule encoder (halo2-gpu_b200/rules.py)."""
import importlib.util
import os
import sys

_PATH = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "halo2-gpu_b200", "rules.py")
_spec = importlib.util.spec_from_file_location("h2b_rules", _PATH)
_mod = importlib.util.module_from_spec(_spec)
sys.modules.setdefault("h2b_rules", _mod)
_spec.loader.exec_module(_mod)
globals().update({k: v for k, v in vars(_mod).items() if not k.startswith("__")})
