"""arcos_b200 — B200 (sm_100a) implementation of the arcos CDR density update.

Host-side mirror of the reference interface (cdr.c / reaction.c entry points
and the rz_array / cdr_grid_t storage) over the C-ABI library
``arcos_b200/libarcos_cdr.so`` (declared in include/arcos_cdr.h).
"""
from .model import KineticModel, Params, Reaction, Species, minimal_model  # noqa: F401
from .grids import GridSpec  # noqa: F401
from .react_table import ReactTable, react_table_read, write_react_table  # noqa: F401
