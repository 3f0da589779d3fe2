/* oracle/shim/sepConfig.h -- stands in for the header SEPlib's cmake step
 * generates from external/SEP/src/sepConfig.h.in, for a Linux/glibc host.
 * TEST INFRASTRUCTURE ONLY: it lets the reference's IO.hpp (included by
 * nlsolver.cpp) compile for the CPU oracle; no SEPlib routine runs (the SEP
 * I/O entry points the solver could reach are aborting stubs in sep_stub.c). */
#pragma once
#define DEFAULT_DOC_PATH ""
#define VPLOT_FONT_DIR ""
#define HAVE_TERMIOS_H 1
#define HAVE_STDIO_H 1
#define HAVE_STDLIB_H 1
#define HAVE_STRING_H 1
#define HAVE_STRINGS_H 1
#define HAVE_SYS_IOCTL_H 1
#define HAVE_SYS_STAT 1
#define HAVE_SYS_FILE_H 1
#define HAVE_SYS_STAT_H 1
#define HAVE_SYS_UIO_H 1
#define HAVE_SIGNAL_H 1
#define HAVE_SYS_TYPES_H 1
#define HAVE_SYS_UTSNAME_H 1
#define HAVE_SYS_PARAM_H 1
#define HAVE_UNISTD_H 1
#define HAVE_FCNTL_H 1
#define HAVE_DIRENT_H 1
#define HAVE_LIMITS_H 1
#define HAVE_ERRNO_H 1
#define HAVE_SYS_SOCKET_H 1
#define HAVE_CTYPE_H 1
#define HAVE_UTIME_H 1
