"""Field export (gridfoam ``io/``): VTU files, written off the step loop."""

from gridfoam_b200.io.vtu import (
    AsyncVtuExporter,
    UnstructuredGrid,
    save_export_fields_as_vtu,
    to_unstructured_grid,
    update_export_cell_data,
)

__all__ = [
    "AsyncVtuExporter",
    "UnstructuredGrid",
    "save_export_fields_as_vtu",
    "to_unstructured_grid",
    "update_export_cell_data",
]
