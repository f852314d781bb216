"""CPU oracle for the all-sources heat-method path.

TEST INFRASTRUCTURE ONLY: a restatement of the reference algorithm that the CUDA
engine's results are compared with. Only tests/, __graft_entry__.smoke() and
bench.py's CPU-baseline leg may import it; the product path never does.

Parity is pinned against golden vectors produced by the reference's own code
(fastcw_lean.ConsistentBatchHeatEngine, lean_geometry, core_analysis) on the
same seeded meshes; see tests/golden/make_golden.py.
"""

from .heat import (  # noqa: F401
    HeatOracle,
    build_oracle_library,
    field_health,
    gradient_basis,
    mean_edge_length,
    msd_and_boundary,
    normalized_divergence,
    operators,
    source_geometry,
    field_eval,
    source_metrics,
)
from .intrinsic import intrinsic_delaunay, robust_operators  # noqa: F401
from .samples import (  # noqa: F401
    boundary_area_loss_fraction,
    clean_vertex_samples,
    csr,
    vertex_samples,
)
