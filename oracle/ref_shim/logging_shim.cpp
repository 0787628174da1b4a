// Test infrastructure (oracle): stand-ins for MonkeyGL's Logger and StopWatch
// (core/Logger.h, core/StopWatch.h), whose originals need log4cplus.  Only the
// declared interface is implemented; messages go to stderr when the
// MKREF_LOG environment variable is set, otherwise they are dropped.
#include <stdarg.h>
#include <stdio.h>
#include <stdlib.h>
#include <time.h>
#include <string>

#include "Logger.h"
#include "StopWatch.h"

namespace MonkeyGL {

static bool log_on() { return getenv("MKREF_LOG") != nullptr; }

static void vlog(const char *tag, const char *fmt, va_list ap) {
    if (!log_on()) return;
    fprintf(stderr, "[mkref %s] ", tag);
    vfprintf(stderr, fmt, ap);
    fputc('\n', stderr);
}

void Logger::Init() {}
void Logger::SetLevel(LogLevel) {}
void Logger::Info(const char *format, ...) { va_list ap; va_start(ap, format); vlog("info", format, ap); va_end(ap); }
void Logger::Warn(const char *format, ...) { va_list ap; va_start(ap, format); vlog("warn", format, ap); va_end(ap); }
void Logger::Error(const char *format, ...) { va_list ap; va_start(ap, format); vlog("error", format, ap); va_end(ap); }
std::string Logger::FormatMsg(const char *format, ...) {
    char buf[2048];
    va_list ap;
    va_start(ap, format);
    vsnprintf(buf, sizeof(buf), format, ap);
    va_end(ap);
    return std::string(buf);
}

long long StopWatch::GetMSStamp() {
    struct timespec ts;
    clock_gettime(CLOCK_MONOTONIC, &ts);
    return (long long)ts.tv_sec * 1000 + ts.tv_nsec / 1000000;
}
StopWatch::StopWatch(const char *format, ...) {
    char buf[1024];
    va_list ap;
    va_start(ap, format);
    vsnprintf(buf, sizeof(buf), format, ap);
    va_end(ap);
    m_strMsg = buf;
    m_starttime_ms = GetMSStamp();
}
StopWatch::~StopWatch() {}

}  // namespace MonkeyGL
