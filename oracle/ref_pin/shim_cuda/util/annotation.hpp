// Interface stand-in (test infrastructure): the host/device decoration macro.
#pragma once
#define HOST_DEVICE_FUN __host__ __device__
