// No-op logging header used only when the reference GustANN sources are
// compiled into the checker library (oracle/_ref). The reference includes
// spdlog for log lines only (src/common.hpp:5-17); none of its search
// arithmetic depends on it. Every macro here discards its arguments.
#pragma once
#include <atomic>
#include <memory>
#include <thread>

#define SPDLOG_TRACE(...) ((void)0)
#define SPDLOG_DEBUG(...) ((void)0)
#define SPDLOG_INFO(...) ((void)0)
#define SPDLOG_WARN(...) ((void)0)
#define SPDLOG_ERROR(...) ((void)0)
#define SPDLOG_CRITICAL(...) ((void)0)
