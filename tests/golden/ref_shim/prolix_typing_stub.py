"""Stand-in for ``prolix.typing`` (TEST INFRASTRUCTURE ONLY).

prolix's typing module builds equinox classes that need JAX.  The force-field
files loaded for the fixtures use from it only the packed-row parameter
tuples, restated here with the reference's row layout (prolix
src/prolix/typing.py:75-94 and :157-194: bond rows (length, k), angle rows
(theta0, k)).
"""

from typing import NamedTuple

from jaxtyping import Array, ArrayLike, Bool, Float, Int  # noqa: F401

BOND_IDX_LENGTH = 0
BOND_IDX_K = 1
ANGLE_IDX_THETA0 = 0
ANGLE_IDX_K = 1

BondIndices = AngleIndices = object


class BondParams(NamedTuple):
  length: object
  k: object

  @classmethod
  def from_row(cls, row):
    return cls(length=row[BOND_IDX_LENGTH], k=row[BOND_IDX_K])


class AngleParams(NamedTuple):
  theta0: object
  k: object

  @classmethod
  def from_row(cls, row):
    return cls(theta0=row[ANGLE_IDX_THETA0], k=row[ANGLE_IDX_K])
