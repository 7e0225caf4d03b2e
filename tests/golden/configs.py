"""The two single-case workloads of the path (defined in bowshock_b200/configs.py; the oracle's copies come from
tests/golden/sweep_oracle.oracle_case)."""
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "..", ".."))

from bowshock_b200.configs import CONFIGS, D_NOSE, config0_case, config1_case  # noqa: E402,F401
