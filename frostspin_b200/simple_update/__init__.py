from .simple_update import SimpleUpdate, UpdateSchedule

__all__ = ["SimpleUpdate", "UpdateSchedule"]
