/* Minimal stand-in for the Yorick API header, used only to compile the
 * reference LongFessler2D.c into the test oracle.  The only Yorick routine
 * that file calls is ypush_long (from its Y_getpid builtin). */
#ifndef ORACLE_STUB_YAPI_H
#define ORACLE_STUB_YAPI_H 1
extern void ypush_long(long value);
#endif
