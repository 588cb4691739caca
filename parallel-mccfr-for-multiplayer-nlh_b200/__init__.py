"""B200 MCCFR trainer: C ABI (libmccfr.so) plus a host mirror of the reference's
GPUCFRTrainer.  The package directory name is not a Python identifier; load it
with `load_package()` from `__graft_entry__`, bench.py or tests/conftest.py,
which register it as `mccfr_b200`.
"""
from . import lib  # noqa: F401
from .trainer import GPUCFRTrainer, Batch, batch_round  # noqa: F401
from .lib import MccfrError, Config, preset, hand_table, generate_hand_table  # noqa: F401
