"""Per-step diagnostics (gridfoam ``post/diagnostics``): continuity error and
solver statistics streamed to CSV without a host round trip per step."""

from gridfoam_b200.post.diagnostics.collector import DiagnosticsCollector
from gridfoam_b200.post.diagnostics.continuity import compute_continuity_error

__all__ = ["DiagnosticsCollector", "compute_continuity_error"]
