/* Minimal GLib / GObject surface needed to compile the reference's task sources
 * (filter, backproject, general-backproject, lamino-backproject,
 * stacked-backproject) and its common/ helpers on a machine without glib.
 * Types carry only what those sources touch; the functions live in
 * ref_glib.cpp and ref_runtime.cpp.  Test infrastructure only. */
#ifndef REFSHIM_GLIB_H
#define REFSHIM_GLIB_H
#include <float.h>
#include <stddef.h>
#include <limits.h>
#include <math.h>
#include <stdarg.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#ifdef __cplusplus
extern "C" {
#endif
typedef float gfloat;
typedef double gdouble;
typedef int gint;
typedef unsigned int guint;
typedef long glong;
typedef unsigned long gulong;
typedef unsigned char guchar;
typedef unsigned short gushort;
typedef int gboolean;
typedef size_t gsize;
typedef ptrdiff_t gssize;
typedef void *gpointer;
typedef const void *gconstpointer;
typedef char gchar;
typedef unsigned long GType;
#define TRUE 1
#define FALSE 0
#define G_PI 3.1415926535897932384626433832795028841971693993751
#define G_MAXFLOAT FLT_MAX
#define G_MAXDOUBLE DBL_MAX
#define G_MAXUINT UINT_MAX
#define G_MAXINT INT_MAX
#define G_MININT INT_MIN
#define G_MAXULONG ULONG_MAX
#define G_BEGIN_DECLS
#define G_END_DECLS
#ifndef MIN
#define MIN(a, b) (((a) < (b)) ? (a) : (b))
#endif
#ifndef MAX
#define MAX(a, b) (((a) > (b)) ? (a) : (b))
#endif
#ifndef ABS
#define ABS(a) (((a) < 0) ? -(a) : (a))
#endif

/* fundamental type ids (values only need to be distinct) */
#define G_TYPE_INVALID ((GType)0)
#define G_TYPE_BOOLEAN ((GType)20)
#define G_TYPE_INT ((GType)24)
#define G_TYPE_UINT ((GType)28)
#define G_TYPE_LONG ((GType)32)
#define G_TYPE_ULONG ((GType)36)
#define G_TYPE_ENUM ((GType)48)
#define G_TYPE_FLOAT ((GType)56)
#define G_TYPE_DOUBLE ((GType)60)
#define G_TYPE_STRING ((GType)64)
#define G_TYPE_BOXED ((GType)72)
#define G_TYPE_VALUE_ARRAY ((GType)100)

typedef struct {
    GType g_type;
    union {
        int i;
        unsigned u;
        float f;
        double d;
        long l;
        unsigned long ul;
        void *p;
        const char *s;
    } data;
} GValue;
#define G_VALUE_INIT {0, {0}}
#define g_value_init(gv, t) ((gv)->g_type = (t), (gv)->data.d = 0, (gv))
#define g_value_unset(gv) ((void)(gv))
#define g_value_get_enum(gv) ((gv)->data.i)
#define g_value_set_enum(gv, x) ((gv)->data.i = (x))
#define g_value_get_int(gv) ((gv)->data.i)
#define g_value_set_int(gv, x) ((gv)->data.i = (x))
#define g_value_get_float(gv) ((gv)->data.f)
#define g_value_set_float(gv, x) ((gv)->data.f = (x))
#define g_value_get_double(gv) ((gv)->data.d)
#define g_value_set_double(gv, x) ((gv)->data.d = (x))
#define g_value_get_uint(gv) ((gv)->data.u)
#define g_value_set_uint(gv, x) ((gv)->data.u = (x))
#define g_value_get_ulong(gv) ((gv)->data.ul)
#define g_value_set_ulong(gv, x) ((gv)->data.ul = (x))
#define g_value_get_string(gv) ((gv)->data.s)
#define g_value_get_boxed(gv) ((gv)->data.p)
#define g_value_set_boxed(gv, x) ((gv)->data.p = (void *)(x))
#define g_value_get_boolean(gv) ((gv)->data.i)
#define g_value_set_boolean(gv, x) ((gv)->data.i = (x))
void g_value_transform(const GValue *src, GValue *dest);

typedef struct {
    guint n_values;
    GValue *values;
    guint n_prealloced;
} GValueArray;
GValueArray *g_value_array_new(guint n_prealloced);
GValueArray *g_value_array_copy(const GValueArray *a);
void g_value_array_free(GValueArray *a);
GValueArray *g_value_array_append(GValueArray *a, const GValue *v);
GValueArray *g_value_array_insert(GValueArray *a, guint index, const GValue *v);
GValue *g_value_array_get_nth(GValueArray *a, guint index);

/* memory */
#define g_malloc(n) malloc((n) ? (n) : 1)
#define g_malloc0(n) calloc(1, (n) ? (n) : 1)
#define g_realloc(p, n) realloc((p), (n))
#define g_free(p) free((void *)(p))
#define g_new(T, n) ((T *)malloc(sizeof(T) * (n)))
#define g_new0(T, n) ((T *)calloc((n) ? (n) : 1, sizeof(T)))

/* strings */
gchar *g_strdup(const gchar *s);
gchar *g_strdup_printf(const gchar *fmt, ...);
gchar *g_strconcat(const gchar *first, ...);
gchar *g_strnfill(gsize length, gchar c);
gchar *g_stpcpy(gchar *dest, const gchar *src);
gint g_strcmp0(const gchar *a, const gchar *b);
gchar **g_strsplit(const gchar *s, const gchar *delim, gint max_tokens);
void g_strfreev(gchar **v);
#define g_snprintf snprintf
#define g_printf printf
#define g_sprintf sprintf

/* regular expressions (only replace_literal is used) */
typedef struct _GRegex GRegex;
GRegex *g_regex_new(const gchar *pattern, int compile_options, int match_options, void *error);
gchar *g_regex_replace_literal(GRegex *re, const gchar *string, gssize len, gint start, const gchar *replacement,
                               int match_options, void *error);
void g_regex_unref(GRegex *re);

/* hash tables with string keys */
typedef struct _GHashTable GHashTable;
guint g_str_hash(gconstpointer v);
gboolean g_str_equal(gconstpointer a, gconstpointer b);
GHashTable *g_hash_table_new(guint (*hash)(gconstpointer), gboolean (*equal)(gconstpointer, gconstpointer));
gboolean g_hash_table_insert(GHashTable *t, gpointer key, gpointer value);
gpointer g_hash_table_lookup(GHashTable *t, gconstpointer key);
void g_hash_table_destroy(GHashTable *t);

/* logging and assertions */
#define G_LOG_LEVEL_ERROR (1 << 2)
#define G_LOG_LEVEL_CRITICAL (1 << 3)
#define G_LOG_LEVEL_WARNING (1 << 4)
#define G_LOG_LEVEL_MESSAGE (1 << 5)
#define G_LOG_LEVEL_INFO (1 << 6)
#define G_LOG_LEVEL_DEBUG (1 << 7)
void g_log(const gchar *domain, int level, const gchar *fmt, ...);
void g_warning(const gchar *fmt, ...);
#define g_debug(...) ((void)0)
#define g_message(...) ((void)0)
#define g_assert(expr) do { if (!(expr)) { fprintf(stderr, "refshim: assertion %s failed\n", #expr); abort(); } } while (0)
#define g_assert_true(expr) g_assert(expr)
#define g_return_val_if_fail(expr, val) do { if (!(expr)) return (val); } while (0)
#define g_return_if_fail(expr) do { if (!(expr)) return; } while (0)

/* errors */
typedef struct { int domain, code; char message[512]; } GError;
void g_set_error(GError **err, int domain, int code, const char *fmt, ...);
void g_set_error_literal(GError **err, int domain, int code, const char *message);

/* GObject */
typedef struct { int dummy; } GParamSpec;
typedef struct { int value; const char *value_name; const char *value_nick; } GEnumValue;
typedef struct _GObject { void *dummy; } GObject;
typedef struct {
    void (*finalize)(GObject *);
    void (*set_property)(GObject *, guint, const GValue *, GParamSpec *);
    void (*get_property)(GObject *, guint, GValue *, GParamSpec *);
} GObjectClass;
#define G_PARAM_READWRITE 3
GParamSpec *refshim_pspec(void);
#define g_param_spec_enum(...) refshim_pspec()
#define g_param_spec_float(...) refshim_pspec()
#define g_param_spec_double(...) refshim_pspec()
#define g_param_spec_uint(...) refshim_pspec()
#define g_param_spec_int(...) refshim_pspec()
#define g_param_spec_boolean(...) refshim_pspec()
#define g_param_spec_string(...) refshim_pspec()
#define g_param_spec_value_array(...) refshim_pspec()
#define g_enum_register_static(name, values) ((GType)(values != NULL))
#define g_object_class_install_property(oclass, id, pspec) ((void)(oclass), (void)(id), (void)(pspec))
#define g_type_class_add_private(klass, size) ((void)(klass), (void)(size))
#define G_OBJECT_WARN_INVALID_PROPERTY_ID(obj, id, pspec) ((void)(obj), (void)(id), (void)(pspec))
void *g_object_new(GType type, ...);
/* Only "num_processed" (a guint, the ufo-core task node's count of inputs
 * processed so far) is answered; the driver sets it before each call. */
void g_object_get(gpointer obj, const gchar *first, ...);
#define g_object_ref(o) (o)
#define g_object_unref(o) ((void)(o))
#define G_OBJECT_CLASS(k) ((GObjectClass *)(k))
#define G_TYPE_CHECK_INSTANCE_CAST(obj, type, ctype) ((ctype *)(obj))
#define G_TYPE_CHECK_INSTANCE_TYPE(obj, type) ((obj) != NULL)
#define G_TYPE_CHECK_CLASS_CAST(k, type, ctype) ((ctype *)(k))
#define G_TYPE_CHECK_CLASS_TYPE(k, type) ((k) != NULL)
#define G_TYPE_INSTANCE_GET_CLASS(obj, type, ctype) ((ctype *)NULL)
#define G_IMPLEMENT_INTERFACE(iface_type, init)
extern guint refshim_num_processed;
#ifdef __cplusplus
}
#endif
#endif
