/* Test infrastructure: the reference includes its configure-generated header
   both as "config.h" and as "include/config.h"; both resolve to the settings
   in oracle/ref/config.h. */
#include "../config.h"
