"""torch.autograd binding of the adjoint sweep.

``expectation(theta)`` returns <psi(theta)|H|psi(theta)> as a differentiable torch scalar.
Its backward is the engine's adjoint sweep (qsv_adjoint): one forward pass, H|psi>, and one
reverse pass over the gates accumulate every parameter's gradient in FP64, as the
reference's run_gradient does on the CPU (src/qarpx/src/simulator/qarp_simulator.cpp:1519-1605).
PyTorch only carries the gradient; the arithmetic is the CUDA kernels'.
"""
from __future__ import annotations

from typing import Sequence

import numpy as np
import torch

from .ir import pack
from .observable import to_masks


class _AdjointExpectation(torch.autograd.Function):
    @staticmethod
    def forward(ctx, theta: torch.Tensor, sim, commands, n_qubits, masks, param_order):
        values = dict(zip(param_order, theta.detach().to("cpu", torch.float64).tolist()))
        if theta.requires_grad:
            stream = pack(commands, values, param_order)
            reg = sim.register(n_qubits)
            reg.reset()
            energy, grad = reg.adjoint(stream, len(param_order), masks)
            ctx.save_for_backward(torch.as_tensor(grad, dtype=theta.dtype, device=theta.device))
        else:
            reg = sim.register(n_qubits)
            reg.reset()
            reg.apply(pack(commands, values))
            energy = reg.expectation(masks).real
        return torch.as_tensor(energy, dtype=theta.dtype, device=theta.device)

    @staticmethod
    def backward(ctx, grad_out):
        (grad,) = ctx.saved_tensors
        return grad_out * grad, None, None, None, None, None


class AdjointExpectation:
    """Differentiable <H> of a parametrised command stream on a B200Simulator."""

    def __init__(self, sim, commands, n_qubits: int, observable, param_order: Sequence[str]):
        self.sim = sim
        self.commands = list(commands)
        self.n_qubits = int(n_qubits)
        self.masks = to_masks(observable, n_qubits, where="run_gradient")
        self.param_order = list(param_order)

    def __call__(self, theta: torch.Tensor) -> torch.Tensor:
        if theta.ndim != 1 or theta.shape[0] != len(self.param_order):
            raise ValueError(f"theta must have shape ({len(self.param_order)},)")
        return _AdjointExpectation.apply(theta, self.sim, self.commands, self.n_qubits, self.masks,
                                         self.param_order)


def expectation(sim, commands, n_qubits, observable, param_order, theta: torch.Tensor) -> torch.Tensor:
    return AdjointExpectation(sim, commands, n_qubits, observable, param_order)(theta)


def parameter_shift(sim, commands, n_qubits, observable, param_order, theta) -> np.ndarray:
    """The reference's parameter-shift rule on the same engine: for every parameter and every
    gate occurrence carrying it, two energy evaluations at +-pi/2 (Pauli rotations: shift
    rule exact for exp(-i t/2 P)), weighted by the occurrence's affine coefficient
    (reference: src/qarp/engines/_gradients.py:258-291, 407-421).  Counterpart of the
    adjoint for the speed comparison; supports one-parameter Pauli-rotation gates."""
    from .ir import Command, GateType as G, affine_coefficients

    masks = to_masks(observable, n_qubits, where="run_gradient")
    values = dict(zip(param_order, [float(v) for v in theta]))
    index = {n: i for i, n in enumerate(param_order)}
    cmds = list(commands)
    concrete = [Command(c.gate, c.qubits, tuple(float(p.evaluate(values)) if hasattr(p, "evaluate")
                                                else float(p) for p in c.params), c.unitary)
                for c in cmds]
    reg = sim.register(n_qubits)
    grad = np.zeros(len(param_order))
    rot = {G.Rx, G.Ry, G.Rz, G.RXX, G.RYY, G.RZZ}
    for i, c in enumerate(cmds):
        for p in c.params:
            for name, alpha in affine_coefficients(p).items():
                if name not in index:
                    continue
                if c.gate not in rot:
                    raise ValueError("parameter_shift here supports Pauli-rotation gates only")
                e = []
                for s in (np.pi / 2, -np.pi / 2):
                    shifted = list(concrete)
                    shifted[i] = Command(c.gate, c.qubits, (concrete[i].params[0] + s,))
                    reg.reset()
                    reg.apply(pack(shifted))
                    e.append(reg.expectation(masks).real)
                grad[index[name]] += alpha * 0.5 * (e[0] - e[1])
    return grad
