/* glibc >= 2.32 removed <sys/sysctl.h>; the reference only includes it. */
