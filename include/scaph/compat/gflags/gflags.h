// Minimal stand-in for <gflags/gflags.h> as the reference's applications use
// it (app/sssp.cu:4,8-9, app/wcc.cu:6,8): DECLARE_* names a FLAGS_<name>
// global that scaph/compat/app.cuh defines; DEFINE_* defines a new one.
// Command-line parsing is done by App's constructor (--name=value).
#ifndef SCAPH_COMPAT_GFLAGS_H
#define SCAPH_COMPAT_GFLAGS_H

#include <string>

#define DECLARE_int32(name) extern int FLAGS_##name
#define DECLARE_int64(name) extern long long FLAGS_##name
#define DECLARE_bool(name) extern bool FLAGS_##name
#define DECLARE_double(name) extern double FLAGS_##name
#define DECLARE_string(name) extern std::string FLAGS_##name

#define DEFINE_int32(name, value, help) int FLAGS_##name = (value)
#define DEFINE_int64(name, value, help) long long FLAGS_##name = (value)
#define DEFINE_bool(name, value, help) bool FLAGS_##name = (value)
#define DEFINE_double(name, value, help) double FLAGS_##name = (value)
#define DEFINE_string(name, value, help) std::string FLAGS_##name = (value)

#endif
