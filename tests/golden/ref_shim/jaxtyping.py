"""Stand-in for jaxtyping: subscriptable placeholders (TEST INFRASTRUCTURE ONLY)."""


class _Any:
  def __getitem__(self, _):
    return object

  def __call__(self, *a, **k):
    return object


Array = object
ArrayLike = object
PRNGKeyArray = object
Float = _Any()
Int = _Any()
Bool = _Any()
UInt = _Any()
Shaped = _Any()
