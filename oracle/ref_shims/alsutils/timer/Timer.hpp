// Plumbing shim: timers are compiled out.
#pragma once
#define ALSVINN_TIME_BLOCK(...)
