"""
The solver contract that sailfish's driver programs against
(sailfish/solver_base.py:8-128).
"""

from abc import ABC, abstractmethod


class SolverBase(ABC):
    @property
    @abstractmethod
    def solution(self):
        """The state written to checkpoints and passed back on restart."""

    @property
    @abstractmethod
    def primitive(self):
        """Primitive data for plotting (may be None)."""

    @property
    @abstractmethod
    def time(self):
        """The simulation time."""

    @property
    @abstractmethod
    def options(self) -> dict:
        """Solver options as a dict."""

    @property
    @abstractmethod
    def physics(self) -> dict:
        """Physics parameters as a dict."""

    @property
    def recommended_cfl(self):
        return self.maximum_cfl

    @property
    @abstractmethod
    def maximum_cfl(self):
        """Largest CFL number the solver supports."""

    @abstractmethod
    def maximum_wavespeed(self):
        """Largest signal speed on the grid."""

    @abstractmethod
    def advance(self, dt):
        """Advance the state by one iteration of size dt."""

    def reductions(self):
        """Diagnostics of the current state; optional."""
