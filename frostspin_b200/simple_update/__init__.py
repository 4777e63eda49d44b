from .simple_update import SimpleUpdate, UpdateSchedule
from .symmetrized_simple_update import SymmetrizedSimpleUpdate

__all__ = ["SimpleUpdate", "SymmetrizedSimpleUpdate", "UpdateSchedule"]
