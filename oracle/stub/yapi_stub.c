/* No-op definition of the single Yorick routine referenced by the reference
 * LongFessler2D.c (its Y_getpid builtin is never called by the oracle). */
void ypush_long(long value) { (void)value; }
