"""Assembly."""

from bempp.assembly import boundary  # noqa: F401
