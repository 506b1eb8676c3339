"""tinker-hp_b200: B200-native AMOEBA induced-dipole polarization path."""
from . import params, water  # noqa: F401
