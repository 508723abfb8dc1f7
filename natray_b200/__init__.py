"""natray_b200: natray's simulation step on B200 (sm_100a), behind the C ABI of include/natray.h."""
from .world import Params, World, build_world, sized_for  # noqa: F401
