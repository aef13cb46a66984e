"""B200-native critical-point tracking (the SimplicialEngine<T,
CriticalPointPredicate<M,T>> path of hguo/ftk2), driven through the C ABI in
include/ftk2b.h.  See ftk2_b200.api for the Python binding."""
from .api import (  # noqa: F401
    Context, CriticalPointPredicate, ExtrudedSimplicialMesh, Ftk2bError, RegularSimplicialMesh,
    SimplicialEngine, UnstructuredSimplicialMesh, field_desc, extruded_mesh_desc, load_library,
    params, regular_mesh_desc, simplex_count,
)
