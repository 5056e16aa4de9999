"""Front-end propagators: ``PauliPropagator`` and ``MajoranaPropagator`` on the B200 engine.

Same public surface as the reference's ``src/monoprop/{monomial,pauli,majorana}_propagator.py`` for the
Heisenberg propagate path: construction from an operator and a reference state with ``cutoff``,
``lower_atol``, ``upper_atol`` (and ``cutoff_type`` for Majorana), ``from_circuit``, ``propagate``,
``expectation_value`` / ``expval``, ``expectation_value_and_gradient``, ``evolved_operator``, ``size`` and
the truncation properties. They drive the ``_core`` module's per-tier classes, like the reference's
front-end drives its ``_core`` through ``_dispatch.dispatch(num_modes)``.
"""

from __future__ import annotations

from collections.abc import Sequence

import numpy as np

from . import _core
from .circuit import Circuit, expand_monomials
from .operators import MajoranaOperator, Pauli, PauliOperator


def dispatch(num_modes: int):
    """The ``_core`` class of the 32-mode storage tier holding ``num_modes`` (``tools/generate-dispatch.py``)."""
    if num_modes < 1 or num_modes > _core.MAX_NUM_MODES:
        raise ValueError(f"num_modes must be in [1, {_core.MAX_NUM_MODES}]; got {num_modes}")
    tier = ((num_modes + 31) // 32) * 32
    return getattr(_core, f"MonomialPropagator{tier:03d}")


class MonomialPropagator:
    """Shared implementation of the two front-ends (``monomial_propagator.py:58-627``)."""

    def _init_simulator(self, terms: dict, num_modes: int, initial_state, *, cutoff: int, cutoff_type: str,
                        lower_atol, upper_atol, basis: str, schrodinger_cutoff=None, basis_change=None,
                        comm=None) -> None:
        self._system_size = num_modes
        self._initial_state = list(initial_state)
        self._simulator = dispatch(num_modes)(initial_operator=terms, cutoff=cutoff,
                                              initial_state=list(initial_state), comm=comm,
                                              schrodinger_cutoff=schrodinger_cutoff, lower_atol=lower_atol,
                                              upper_atol=upper_atol, cutoff_type=cutoff_type,
                                              basis_change=basis_change, logical_num_modes=num_modes, basis=basis)

    @classmethod
    def from_circuit(cls, circuit: Circuit, initial_operator, **config):
        """Construct with the circuit's initial state and propagate it (``monomial_propagator.py:133-151``)."""
        p = cls(initial_operator, list(circuit.initial_state), **config)
        p.propagate(circuit)
        return p

    def _check_circuit(self, circuit: Circuit) -> None:
        if circuit._state_given and sorted(circuit.initial_state) != sorted(self._initial_state):
            raise ValueError(f"circuit.initial_state {list(circuit.initial_state)} does not match the propagator's "
                             f"initial state {list(self._initial_state)}. Construct the propagator with this "
                             "circuit's initial state (or via from_circuit).")
        if circuit.system_size != self._system_size:
            raise ValueError(f"Circuit system_size={circuit.system_size} does not match propagator width "
                             f"{self._system_size}.")

    def propagate(self, circuit: Circuit, *, only_rotate_len_k: int | None = None) -> None:
        """Evolve and contract immediately (Heisenberg: gates applied last to first)."""
        if only_rotate_len_k is not None and not 0 < only_rotate_len_k <= 2 * self._system_size:
            raise ValueError(f"only_rotate_len_k={only_rotate_len_k} is out of range; must be 0 < k <= 2*num_qubits ")
        self._check_circuit(circuit)
        gates = self._circuit_gates(circuit)
        monos, g, mapping, _ = expand_monomials(gates, circuit.resolved_mapping, self._system_size)
        params = [float(v) for v in circuit.parameters]
        if monos and not params:
            raise ValueError("propagate() needs a circuit with bound parameters.")
        self._simulator.propagate([list(m) for m in monos], mapping, g, params, only_rotate_len_k)

    def build_graph(self, circuit: Circuit, *, seed_parameters=None, only_rotate_len_k: int | None = None) -> None:
        """Keep the circuit's truncation structure, built at ``seed_parameters`` (default: the circuit's
        own), for evaluation at other parameters (``monomial_propagator.py:201-255``)."""
        self._check_circuit(circuit)
        gates = self._circuit_gates(circuit)
        monos, g, mapping, gidx = expand_monomials(gates, circuit.resolved_mapping, self._system_size)
        seed = circuit.parameters if seed_parameters is None else seed_parameters
        self._simulator.build_graph([list(m) for m in monos], mapping, g, gidx, self._bind(seed) or None,
                                    only_rotate_len_k)
        self._n_params = circuit.n_parameters

    @property
    def n_parameters(self) -> int:
        return getattr(self, "_n_params", 0)

    def graph_layers(self) -> int:
        return self._simulator.graph_layers()

    def contract_partially(self, parameters=None, *, inplace: bool = True) -> np.ndarray:
        """The stored graph replayed at ``parameters`` as raw coefficients (store order, core term
        excluded); ``inplace`` consumes the graph (``monomial_propagator.py:478-510``)."""
        coeffs = np.asarray(self._simulator.contract_partially(self._bind(parameters), inplace))
        if inplace:
            self._n_params = 0
        return coeffs

    def gradient(self, parameters=None):
        return self.expectation_value_and_gradient(parameters)[1]

    def expectation_value_functional(self, pare_threshold: float | None = None):
        """A reusable callable ``parameters -> <O>`` over the stored graph; with ``pare_threshold`` the graph
        is pared of what cannot reach the reference state (``monomial_propagator.py:380-401``). It goes
        stale (RuntimeError when called) after build_graph, contract_partially or update_initial_operator."""
        fn = self._simulator.expectation_value_functional(pare_threshold)
        return lambda parameters=None: fn(self._bind(parameters))

    def expectation_value_and_gradient_functional(self, pare_threshold: float | None = None):
        """Like :meth:`expectation_value_functional`, returning ``(<O>, gradient)``
        (``monomial_propagator.py:403-428``)."""
        fn = self._simulator.expectation_value_and_gradient_functional(pare_threshold)

        def _call(parameters=None):
            value, grad = fn(self._bind(parameters))
            return value, np.asarray(grad, dtype=np.float64)

        return _call

    @property
    def parameter_mapping(self) -> list[int]:
        """Parameter index of every graph layer (``monomial_propagator.py:303-335``); assignable, per layer
        or per gate, to re-wire the stored graph's parameters."""
        return list(self._simulator.parameter_mapping)

    @parameter_mapping.setter
    def parameter_mapping(self, mapping) -> None:
        resolved = [int(i) for i in mapping]
        self._simulator.parameter_mapping = resolved
        self._n_params = max(self._simulator.parameter_mapping, default=-1) + 1

    def n_gates(self) -> int:
        return self._simulator.n_gates()

    def graph_size(self) -> tuple[int, int]:
        """(cos-only indices, pairs) of the stored graph (``monomial_propagator.py:560-568``)."""
        return tuple(self._simulator.graph_size())

    def operator_memory_breakdown(self) -> dict:
        return dict(self._simulator.operator_memory_breakdown())

    def __deepcopy__(self, memo):
        import copy

        new = self.__class__.__new__(self.__class__)
        for k, v in self.__dict__.items():
            new.__dict__[k] = v.__deepcopy__(memo) if k == "_simulator" else copy.deepcopy(v, memo)
        return new

    expval_functional = expectation_value_functional
    expval_and_grad_functional = expectation_value_and_gradient_functional
    grad = gradient

    def expectation_value(self, parameters=None) -> float:
        return self._simulator.expectation_value(self._bind(parameters))

    def expectation_value_and_gradient(self, parameters=None):
        return self._simulator.expectation_value_and_gradient(self._bind(parameters))

    expval = expectation_value
    expval_and_grad = expectation_value_and_gradient

    def size(self) -> int:
        return self._simulator.size()

    @property
    def num_modes(self) -> int:
        return self._system_size

    @property
    def cutoff(self) -> int:
        return self._simulator.cutoff

    @cutoff.setter
    def cutoff(self, value: int) -> None:
        self._simulator.cutoff = value

    @property
    def lower_atol(self):
        return self._simulator.lower_atol

    @lower_atol.setter
    def lower_atol(self, value) -> None:
        self._simulator.lower_atol = value

    @property
    def upper_atol(self):
        return self._simulator.upper_atol

    @upper_atol.setter
    def upper_atol(self, value) -> None:
        self._simulator.upper_atol = value

    @property
    def cutoff_type(self) -> str:
        return self._simulator.cutoff_type

    @property
    def schrodinger(self) -> bool:
        return self._simulator.schrodinger

    @staticmethod
    def _bind(parameters) -> list[float]:
        if parameters is None:
            return []
        return [float(v) for v in np.asarray(parameters, dtype=np.float64).reshape(-1)]


class PauliPropagator(MonomialPropagator):
    """Qubit propagator; ``cutoff`` is the maximum Pauli weight (``pauli_propagator.py:44-86``)."""

    def __init__(self, initial_operator: PauliOperator, initial_state: Sequence[int], *, cutoff: int,
                 schrodinger_cutoff: int | None = None, lower_atol: float | None = None,
                 upper_atol: float | None = None, comm=None) -> None:
        self._init_simulator(initial_operator.get_local_operator().terms, initial_operator.num_qubits, initial_state,
                             cutoff=cutoff, cutoff_type="support", lower_atol=lower_atol, upper_atol=upper_atol,
                             basis="pauli", schrodinger_cutoff=None if schrodinger_cutoff is None
                             else 2 * schrodinger_cutoff, comm=comm)

    @property
    def num_qubits(self) -> int:
        return self._system_size

    def _circuit_gates(self, circuit: Circuit):
        if circuit.family == "majorana":
            raise TypeError("PauliPropagator requires a qubit circuit; its gates are Majorana/fermionic. Use "
                            "MajoranaPropagator for those.")
        return circuit.gates

    def evolved_operator(self, parameters=None, *, atol: float = 1e-12) -> PauliOperator:
        raw = self._simulator.evolved_operator(self._bind(parameters), atol)
        terms = {Pauli.from_slots(slots): complex(c) for slots, c in raw.items()}
        return PauliOperator(terms, self.num_qubits)

    def update_initial_operator(self, new_operator: PauliOperator) -> None:
        """Re-weight the initial operator: its terms must already be stored (``pauli_propagator.py:215-237``)."""
        self._simulator.update_initial_operator(new_operator.get_local_operator().terms)


class MajoranaPropagator(MonomialPropagator):
    """Fermionic propagator over Majorana monomials (``majorana_propagator.py:44-93``)."""

    def __init__(self, initial_operator, initial_state: Sequence[int], *, cutoff: int,
                 schrodinger_cutoff: int | None = None, cutoff_type: str = "length",
                 lower_atol: float | None = None, upper_atol: float | None = None,
                 basis_change: list[list[int]] | None = None, comm=None) -> None:
        op = initial_operator.get_majorana_operator()
        self._init_simulator(op.terms, op.num_modes, initial_state, cutoff=cutoff, cutoff_type=cutoff_type,
                             lower_atol=lower_atol, upper_atol=upper_atol, basis="majorana",
                             schrodinger_cutoff=schrodinger_cutoff, basis_change=basis_change, comm=comm)

    def _circuit_gates(self, circuit: Circuit):
        if circuit.family == "pauli":
            raise TypeError("MajoranaPropagator requires a Majorana/fermionic circuit; its gates are Pauli. Use "
                            "PauliPropagator for those.")
        return circuit.gates

    def evolved_operator(self, parameters=None, *, atol: float = 1e-12) -> MajoranaOperator:
        raw = self._simulator.evolved_operator(self._bind(parameters), atol)
        return MajoranaOperator(raw, self._system_size)

    def update_initial_operator(self, new_operator) -> None:
        """Re-weight the initial operator: its terms must already be stored (``majorana_propagator.py:125-142``)."""
        self._simulator.update_initial_operator(new_operator.get_majorana_operator().terms)

    @property
    def cutoff_type(self) -> str:
        return self._simulator.cutoff_type

    @cutoff_type.setter
    def cutoff_type(self, value: str) -> None:
        self._simulator.cutoff_type = value
