from .classical_c4v import (
    energy_per_bond,
    env_1site,
    env_2sites,
    ising_initial_environment,
    ising_site_tensors,
    iterate_c4v,
)

__all__ = [
    "energy_per_bond",
    "env_1site",
    "env_2sites",
    "ising_initial_environment",
    "ising_site_tensors",
    "iterate_c4v",
]
