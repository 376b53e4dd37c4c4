// Stand-in for the one macro the reference's include/kernel.hpp takes from Cornerstone's
// util/annotation.hpp: host-only compilation needs no decoration.
#pragma once
#define HOST_DEVICE_FUN
