// Replaces the reference's spdlog-backed Logger.cpp (spdlog is an absent
// submodule): every level prints to stderr.
#include "common/Logger.h"
#include <cstdio>
namespace Gyunity {
Logger::Logger() {}
Logger::~Logger() {}
void Logger::Info(const std::string& m) const { std::fprintf(stderr, "%s\n", m.c_str()); }
void Logger::Warn(const std::string& m) const { std::fprintf(stderr, "%s\n", m.c_str()); }
void Logger::Debug(const std::string& m) const { std::fprintf(stderr, "%s\n", m.c_str()); }
void Logger::Error(const std::string& m, bool) const { std::fprintf(stderr, "%s\n", m.c_str()); }
void Logger::Critical(const std::string& m, bool) const { std::fprintf(stderr, "%s\n", m.c_str()); }
void Logger::Flush() const {}
void Logger::SetLevel(const std::string&) {}
int Logger::LevelFromString(const std::string&) { return 0; }
DefaultLogger::DefaultLogger() {}
InfoLogger::InfoLogger() {}
Logger* GetDefaultLogger() { static DefaultLogger l; return &l; }
Logger* GetInfoLogger() { static InfoLogger l; return &l; }
}  // namespace Gyunity
