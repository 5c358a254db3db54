"""Physics executor with the calling convention of the reference
``SparsePhysics`` (``src/neuralpom/hybrid/sparse_physics.py:120-251``).

``advance(core, steps)`` resets the clock bookkeeping exactly like the
reference's no-grad branch (``time0 = time``, ``iint = 0``, ``iend =
steps``) and runs ``core.run_time_loop()`` on the B200 library;
``differentiable=True`` advances in chunks of
``chunk_steps``, each one autograd node whose backward is the CUDA step
adjoint, like the reference's checkpointed chunks.
"""
from __future__ import annotations

import torch

from .core import B200Core, CORE_REGISTRY


class B200Physics:
    def __init__(self, device="cuda", rank=0, chunk_steps=6, core_name="implicit_p0_fixed", **_ignored):
        if core_name not in CORE_REGISTRY:
            raise ValueError(f"Unsupported physics core: {core_name}")
        if chunk_steps < 1:
            raise ValueError("chunk_steps must be positive")
        self.device = torch.device(device)
        if self.device.type != "cuda":
            raise ValueError("the B200 physics runs on CUDA devices only")
        self.global_rank = rank
        self.core_name = core_name
        self.core_cls = CORE_REGISTRY[core_name]
        self.chunk_steps = int(chunk_steps)

    def advance(self, core, steps=6, differentiable=False):
        steps = int(steps)
        if steps < 1:
            raise ValueError("steps must be positive")
        if not isinstance(core, B200Core) or core.core_name != self.core_name:
            raise TypeError(f"B200Physics({self.core_name!r}) requires the matching B200 core")
        if differentiable:
            # chunks of chunk_steps, each one autograd node with a checkpoint
            # per internal step (sparse_physics.py:108-149)
            for start in range(0, steps, self.chunk_steps):
                n = min(self.chunk_steps, steps - start)
                core.time0 = float(core.time)
                core.iint = 0
                core.iend = n
                with torch.enable_grad():
                    core.run_time_loop()
                if core.iint != n:
                    raise RuntimeError("Physical core returned before the checkpoint chunk completed")
            return
        core.time0 = float(core.time)
        core.iint = 0
        core.iend = steps
        with torch.no_grad():
            core.run_time_loop()
        if core.iint != steps:
            raise RuntimeError("Physical core returned before the requested steps completed")
