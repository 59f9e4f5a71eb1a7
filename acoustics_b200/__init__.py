"""B200-native FDTD time-stepping hot path of jhwang7628/acoustics."""
from .scene import *  # noqa: F401,F403
