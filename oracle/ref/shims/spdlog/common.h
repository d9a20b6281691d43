// Stand-in for spdlog/common.h: the reference only forward-declares the logger.
#pragma once
namespace spdlog { class logger; }
