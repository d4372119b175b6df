"""Parameter control systems of netlist circuits.

The reference lets Python scripts adjust circuit parameters between time
steps (flowsolver/src/ControlSystemsManager.cxx:7-52, ParameterController.cxx:
242-410, called once per step after the circuits' finalisation,
itrdrv.f90:2100).  Each script defines a controller with
``updateControl(currentParameterValue, delt, pressures, flows, volumes)``
returning the parameter's new value; the dictionaries hold the circuit's
nodal pressures, component flows and tracked volumes by 1-based index.
Controllers run in ascending priority, and each may publish values for
the ones after it (the broadcast dictionaries).

:class:`ParameterController` is a base class with the method names those
scripts use, so that a script ported to Python 3 runs with little change;
:func:`run_controllers` is the per-step driver the time stepper calls.
"""
from __future__ import annotations

from typing import Dict, Iterable, List, Tuple

import numpy as np


class ParameterController:
    """Base class of a control system: override :meth:`updateControl`.

    ``name`` is the key under which this controller's broadcast values reach
    the others (the reference uses the script's base name);
    ``controllerPriority`` orders the controllers (lower first)."""

    controllerPriority = 0

    def __init__(self, name: str):
        self.name = name
        self._broadcast: Dict[str, float] = {}
        self._received: Dict[str, Dict[str, float]] = {}

    def updateControl(self, currentParameterValue, delt, dictionaryOfPressuresByNodeIndex,
                      dictionaryOfFlowsByComponentIndex, dictionaryOfVolumesByComponentIndex):
        raise NotImplementedError

    def getControllerPriority(self) -> int:
        return self.controllerPriority

    def addBroadcastVariable(self, key: str, value) -> None:
        self._broadcast[key] = value

    def clearBroadcastData(self) -> None:
        self._broadcast = {}

    def getRecievedBroadcastValue(self, controller_name: str, key: str):
        """A value another controller published this step or before (the
        spelling is the reference scripts')."""
        return self._received[controller_name][key]

    def broadcast_data(self) -> Dict[str, Dict[str, float]]:
        return {self.name: dict(self._broadcast)}

    def receive_broadcast(self, data: Dict[str, Dict[str, float]]) -> None:
        self._received = {k: dict(v) for k, v in data.items()}


class PeriodicTableController(ParameterController):
    """The reference's prescribedPeriodicFlow / prescribedPeriodicPressure
    controls (its flowPrescriber / pressurePrescriber scripts): a table of
    (time, value) rows starting at time 0 repeats with the period of its
    last time; each step advances the periodic time by delt (wrapping once
    it reaches the period) and returns the table's linear interpolation
    there."""

    def __init__(self, name: str, times, values):
        super().__init__(name)
        self.times = np.asarray(times, dtype=np.float64)
        self.values = np.asarray(values, dtype=np.float64)
        if self.times.ndim != 1 or self.times.size < 2 or self.times.shape != self.values.shape:
            raise ValueError("a periodic table needs two or more (time, value) rows")
        if self.times[0] != 0.0 or np.any(np.diff(self.times) <= 0.0):
            raise ValueError("periodic table times must start at 0 and increase")
        self.period = float(self.times[-1])
        self.time = 0.0

    @classmethod
    def from_file(cls, name: str, path: str) -> "PeriodicTableController":
        """Two plain-text columns (time, value), as the reference's <name>.dat."""
        data = np.loadtxt(path, ndmin=2)
        return cls(name, data[:, 0], data[:, 1])

    def updateControl(self, currentParameterValue, delt, *observables):
        self.time += delt
        if self.time >= self.period:
            self.time -= self.period
        return float(np.interp(self.time, self.times, self.values))


class BleedController(ParameterController):
    """The reference's built-in bleed control (ParameterController.cxx:
    66-74, timers.cxx): from the trigger step on (1600 steps after the
    start, counted by its own timer) the controlled resistance or compliance
    is set to 0.001.  Built-in controllers update after the Python ones
    (ControlSystemsManager.cxx:7-16), hence the infinite priority."""

    controllerPriority = float("inf")

    def __init__(self, name: str = "bleed", trigger_step: int = 1600, value: float = 0.001):
        super().__init__(name)
        self.step = 0
        self.trigger_step = int(trigger_step)
        self.value = float(value)

    def updateControl(self, currentParameterValue, delt, *observables):
        on = self.step >= self.trigger_step
        self.step += 1
        return self.value if on else currentParameterValue


class LeftVentricularElastanceController(ParameterController):
    """The reference's built-in left-ventricular elastance control
    (ParameterController.cxx:11-57): the time-varying elastance of Pope et
    al., Math. Biosci. Eng. 6 (2009) 93-115 -- a raised cosine from
    ``e_min`` to ``e_max`` over ``t_max``, back down over ``t_relax``, then
    ``e_min`` to the end of the period -- on a periodic time advanced by
    delt each step.  The defaults are the reference's values.  At set-up the
    controlled elastance takes the value at the starting time
    (:meth:`elastance`)."""

    controllerPriority = float("inf")

    def __init__(self, name: str = "lvElastance", start_time: float = 0.0, t_max: float = 0.2782,
                 t_relax: float = 0.1391, e_min: float = 4.10246e-3, e_max: float = 3.0827e-1,
                 period: float = 0.86):
        super().__init__(name)
        self.time = float(start_time)
        self.t_max, self.t_relax, self.e_min, self.e_max, self.period = t_max, t_relax, e_min, e_max, period

    def elastance(self) -> float:
        t, de = self.time, self.e_max - self.e_min
        if t <= self.t_max:
            return self.e_min + 0.5 * de * (1.0 - np.cos(t * np.pi / self.t_max))
        if t <= self.t_max + self.t_relax:
            return self.e_min + 0.5 * de * (1.0 + np.cos((t - self.t_max) * (np.pi / self.t_relax)))
        return self.e_min

    def updateControl(self, currentParameterValue, delt, *observables):
        self.time += delt
        if self.time >= self.period:
            self.time -= self.period
        return float(self.elastance())


def run_controllers(bound: Iterable[Tuple[object, str, int, ParameterController]], delt: float) -> None:
    """One update of every control system (updateAndPassStateInformation-
    BetweenPythonParameterControllers): ``bound`` holds (circuit, target,
    index, controller) with ``circuit`` offering get_parameter /
    set_parameter / observables.  Controllers run in ascending priority
    (ties in the given order); each sees the broadcast values of the ones
    before it, a value published earlier keeping precedence."""
    items: List = sorted(bound, key=lambda b: b[3].getControllerPriority())
    gathered: Dict[str, Dict[str, float]] = {}
    for circuit, target, index, ctl in items:
        ctl.receive_broadcast(gathered)
        p, q, v = circuit.observables()
        new = ctl.updateControl(circuit.get_parameter(target, index), delt, p, q, v)
        circuit.set_parameter(target, index, float(new))
        for k, val in ctl.broadcast_data().items():
            gathered.setdefault(k, val)
