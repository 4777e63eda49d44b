from .classical_c4v import (
    correlation_length,
    edge_transfer_spectrum,
    energy_per_bond,
    env_1site,
    env_2sites,
    ising_initial_environment,
    ising_site_tensors,
    iterate_c4v,
    iterate_c4v_many,
)
from .ctm_environment import CTMEnvironment
from .sequential_ctmrg import SequentialCTMRG
from .simultaneous_ctmrg import SimultaneousCTMRG
from .symmetrized_ctmrg import SymmetrizedCTMRG

__all__ = [
    "CTMEnvironment",
    "SequentialCTMRG",
    "SimultaneousCTMRG",
    "SymmetrizedCTMRG",
    "correlation_length",
    "edge_transfer_spectrum",
    "energy_per_bond",
    "env_1site",
    "env_2sites",
    "ising_initial_environment",
    "ising_site_tensors",
    "iterate_c4v",
    "iterate_c4v_many",
]
