"""nimgpu: B200 (sm_100a) library for the NIM time advance of the
ijarrah2/NIM-CONV22-SHARED solver, reached through the C ABI in
include/nim_gpu.h.  The Python layer only marshals arrays."""
from . import _abi, config
from ._abi import NimError, StepStats, Params, MeshParams
from .mesh import Mesh, temperature_noise, apply_temperature_noise
from .solver import NimSolver, autotune_batch, batch_step, field_len
from .slabs import SlabGroup, SlabRank, exchange_packed, slab_halo, slab_layout

__all__ = ["_abi", "config", "NimError", "StepStats", "Params", "MeshParams", "Mesh",
           "temperature_noise", "apply_temperature_noise", "NimSolver", "autotune_batch", "batch_step", "field_len",
           "SlabGroup", "SlabRank", "exchange_packed", "slab_halo", "slab_layout"]
