"""Shared vocabulary of the GRG matmul path: traversal direction and node-init modes.

The names and string values are the ones the reference package uses
(``pygrgl_spmv/backends/types.py:8-21`` and the parsers at ``:46-78``), so that
specs built by either package compare equal (both enums are ``StrEnum``).
"""

from __future__ import annotations

from enum import StrEnum


class Direction(StrEnum):
    """``up`` maps samples to mutations (X·G); ``down`` maps mutations to samples."""

    UP = "up"
    DOWN = "down"


class InitMode(StrEnum):
    """How node values are initialised before a traversal."""

    NONE = "none"
    XTX = "xtx"
    VECTOR = "vector"
    MATRIX = "matrix"


def parse_direction(direction) -> Direction:
    """Accept ``Direction``, a case-insensitive string, or an enum member named UP/DOWN.

    The last form covers ``pygrgl.TraversalDirection`` without importing pygrgl.
    """
    if isinstance(direction, Direction):
        return direction
    if isinstance(direction, str):
        key = direction.lower()
        if key == "up":
            return Direction.UP
        if key == "down":
            return Direction.DOWN
        raise ValueError(f"Unknown direction {direction!r}; expected up or down")
    name = getattr(direction, "name", None)
    if name == "UP":
        return Direction.UP
    if name == "DOWN":
        return Direction.DOWN
    raise ValueError(
        f"unknown direction: {direction!r}. Expected 'up', 'down', "
        "pygrgl.TraversalDirection.UP, or pygrgl.TraversalDirection.DOWN"
    )


def parse_init_mode(init_mode) -> InitMode:
    if isinstance(init_mode, InitMode):
        return init_mode
    key = str(init_mode).lower()
    for mode in InitMode:
        if mode.value == key:
            return mode
    raise ValueError(f"Unknown init_mode {init_mode!r}; expected one of (none, xtx, vector, matrix)")


__all__ = ["Direction", "InitMode", "parse_direction", "parse_init_mode"]
