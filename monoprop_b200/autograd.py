"""``<0|O(theta)|0>`` as a differentiable torch function of the circuit parameters.

The forward pass runs the engine's propagation with coefficient checkpoints every ``segment_gates``
gates (``mpx_adjoint_forward``); the backward pass is the engine's hand-written adjoint sweep
(``mpx_adjoint_backward``), which replays each segment from its checkpoint and returns
``d<O>/d(angle_l)`` for every layer in one reverse sweep. With ``angle_l = theta[map_l] * g_l``
(``MPFunctions.cpp:57-69``), ``d<O>/d theta_p = sum_{l: map_l = p} g_l d<O>/d angle_l``.

The derivative is that of the frozen-structure surrogate, as in the reference's
``expectation_value_and_gradient`` (``MPFunctions.cpp:207-246``): the truncation decisions taken at
``theta`` are held fixed. PyTorch is used only for the ``torch.autograd.Function`` plumbing; all
arithmetic runs in the CUDA engine.
"""

from __future__ import annotations

import numpy as np
import torch

from . import _native


class _Expectation(torch.autograd.Function):
    @staticmethod
    def forward(ctx, theta: torch.Tensor, prop: DifferentiablePropagation) -> torch.Tensor:
        ev = prop.forward_value(theta.detach().to("cpu", torch.float64).numpy())
        ctx.prop = prop
        ctx.meta = (theta.dtype, theta.device)
        return torch.tensor(ev, dtype=torch.float64, device=theta.device)

    @staticmethod
    def backward(ctx, grad_out: torch.Tensor):
        dtype, device = ctx.meta
        g = torch.from_numpy(ctx.prop.backward_grad()).to(device=device, dtype=dtype)
        return grad_out.to(dtype) * g, None


class DifferentiablePropagation:
    """One observable and circuit on one engine; call it with ``theta`` (a torch tensor of parameters)."""

    def __init__(self, workload, segment_gates: int = 0, device: int = 0):
        self.workload = workload
        self.segment_gates = int(segment_gates)
        self.engine = _native.engine_for(workload, device=device)
        self.map = np.asarray(workload.param_map, dtype=np.int64)
        self.g = np.asarray(workload.gen_coeffs, dtype=np.float64)
        self.n_params = int(self.map.max()) + 1 if self.map.size else 0
        self.circuit = self.engine.upload(workload.gen_words(), workload.angles())
        self._pending = False

    def __call__(self, theta: torch.Tensor) -> torch.Tensor:
        return _Expectation.apply(theta, self)

    def forward_value(self, theta: np.ndarray) -> float:
        theta = np.asarray(theta, dtype=np.float64).reshape(-1)
        if theta.size != self.n_params:
            raise ValueError(f"expected {self.n_params} parameters, got {theta.size}")
        self.circuit.set_angles(theta[self.map] * self.g)
        ev = self.engine.adjoint_forward(self.circuit, self.segment_gates)
        self._pending = True
        return ev

    def backward_grad(self) -> np.ndarray:
        if not self._pending:
            raise RuntimeError("backward needs the forward pass of the same evaluation")
        ga = self.engine.adjoint_backward(self.circuit)
        self._pending = False
        grad = np.zeros(self.n_params, dtype=np.float64)
        np.add.at(grad, self.map, self.g * ga)
        return grad

    def value_and_grad(self, theta) -> tuple[float, np.ndarray]:
        """<O> and d<O>/d theta without autograd (one forward + one adjoint sweep)."""
        ev = self.forward_value(np.asarray(theta, dtype=np.float64))
        return ev, self.backward_grad()

    def close(self) -> None:
        self.circuit.close()
        self.engine.close()
