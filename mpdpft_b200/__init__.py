"""B200-native self-consistent DPFT loop (mpDPFT hot path)."""
from . import abi  # noqa: F401
