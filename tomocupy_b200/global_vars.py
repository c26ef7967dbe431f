"""Process-wide ``args`` / ``params`` namespaces, as in the reference
(src/tomocupy/global_vars.py:43-44).  The operator classes read them the way
the reference's do (e.g. ``BackprojFunctions`` reads ``params.n``)."""
from argparse import Namespace

from .config import make_args

args = make_args()
params = Namespace()


def reset(**overrides) -> None:
    """Reset ``args`` to the defaults plus overrides and clear ``params``."""
    fresh = make_args(**overrides)
    args.__dict__.clear()
    args.__dict__.update(fresh.__dict__)
    params.__dict__.clear()
