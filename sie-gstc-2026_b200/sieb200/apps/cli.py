"""Command-line helpers of the applications, with the reference's parsing rules
and messages (include/sie_mom/utils/cli_helpers.hpp)."""

from __future__ import annotations

import math
import re

INTERIOR, EXTERIOR = 1, 2

# std::stod accepts an optional sign, decimal or exponent forms, inf and nan.
_REAL = re.compile(r"\s*[+-]?((\d+\.?\d*|\.\d+)([eE][+-]?\d+)?|inf(inity)?|nan)", re.IGNORECASE)
_INTEGER = re.compile(r"\s*[+-]?\d+")


def require_value(argv: list[str], index: int) -> tuple[str, int]:
    """The value after argv[index] and the advanced index (require_value)."""
    if index + 1 >= len(argv):
        raise ValueError(f"missing value for option {argv[index]}")
    return argv[index + 1], index + 1


def parse_real(text: str, option: str) -> float:
    m = _REAL.match(text)
    if m is None:
        raise ValueError("stod")
    value = float(m.group(0))
    if m.end() != len(text) or not math.isfinite(value):
        raise ValueError(f"invalid numeric value for {option}: {text}")
    return value


def parse_integer(text: str, option: str) -> int:
    m = _INTEGER.match(text)
    if m is None:
        raise ValueError("stol")
    value = int(m.group(0))
    if m.end() != len(text) or not -2**31 <= value < 2**31:
        raise ValueError(f"invalid integer value for {option}: {text}")
    return value


def parse_region(text: str) -> int:
    if text == "interior":
        return INTERIOR
    if text == "exterior":
        return EXTERIOR
    raise ValueError("source region must be interior or exterior")


def parse_vector(argv: list[str], index: int, option: str) -> tuple[tuple[float, float, float], int]:
    out = []
    for _ in range(3):
        text, index = require_value(argv, index)
        out.append(parse_real(text, option))
    return (out[0], out[1], out[2]), index
