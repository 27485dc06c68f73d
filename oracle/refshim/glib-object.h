/* GLib object layer of the shim (see glib.h).  Test infrastructure only. */
#include <glib.h>
