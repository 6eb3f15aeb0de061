#pragma once
// Oracle build shim: forwards to the fmt copy bundled with spdlog (header-only).
#include <spdlog/fmt/bundled/ranges.h>
