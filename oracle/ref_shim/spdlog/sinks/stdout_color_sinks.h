// Companion of the no-op spdlog header (see ../spdlog.h); intentionally empty.
#pragma once
