// The GLib functions declared in glib.h: value arrays, the string helpers the
// reference's kernel generators use, literal regex replacement, a string-keyed
// hash table and logging.  Test infrastructure only.
#include <regex>
#include <string>
#include <vector>

#include <glib.h>

extern "C" {

guint refshim_num_processed = 0;

void g_value_transform(const GValue *src, GValue *dest)
{
    double v = 0.0;
    switch (src->g_type) {
        case G_TYPE_INT: v = src->data.i; break;
        case G_TYPE_UINT: v = src->data.u; break;
        case G_TYPE_FLOAT: v = src->data.f; break;
        case G_TYPE_DOUBLE: v = src->data.d; break;
        case G_TYPE_ULONG: v = (double)src->data.ul; break;
        case G_TYPE_LONG: v = (double)src->data.l; break;
        default: v = src->data.d; break;
    }
    switch (dest->g_type) {
        case G_TYPE_INT: dest->data.i = (int)v; break;
        case G_TYPE_UINT: dest->data.u = (unsigned)v; break;
        case G_TYPE_FLOAT: dest->data.f = (float)v; break;
        case G_TYPE_ULONG: dest->data.ul = (unsigned long)v; break;
        case G_TYPE_LONG: dest->data.l = (long)v; break;
        default: dest->data.d = v; break;
    }
}

GValueArray *g_value_array_new(guint n_prealloced)
{
    GValueArray *a = (GValueArray *)calloc(1, sizeof(GValueArray));
    a->n_prealloced = n_prealloced ? n_prealloced : 1;
    a->values = (GValue *)calloc(a->n_prealloced, sizeof(GValue));
    return a;
}

static void reserve(GValueArray *a, guint n)
{
    if (n <= a->n_prealloced) return;
    guint cap = a->n_prealloced * 2 > n ? a->n_prealloced * 2 : n;
    a->values = (GValue *)realloc(a->values, cap * sizeof(GValue));
    a->n_prealloced = cap;
}

GValueArray *g_value_array_copy(const GValueArray *src)
{
    GValueArray *a = g_value_array_new(src->n_values);
    memcpy(a->values, src->values, src->n_values * sizeof(GValue));
    a->n_values = src->n_values;
    return a;
}

void g_value_array_free(GValueArray *a)
{
    if (!a) return;
    free(a->values);
    free(a);
}

GValueArray *g_value_array_insert(GValueArray *a, guint index, const GValue *v)
{
    if (index > a->n_values) index = a->n_values;
    reserve(a, a->n_values + 1);
    memmove(a->values + index + 1, a->values + index, (a->n_values - index) * sizeof(GValue));
    if (v)
        a->values[index] = *v;
    else
        memset(a->values + index, 0, sizeof(GValue));
    a->n_values++;
    return a;
}

GValueArray *g_value_array_append(GValueArray *a, const GValue *v) { return g_value_array_insert(a, a->n_values, v); }

GValue *g_value_array_get_nth(GValueArray *a, guint index) { return index < a->n_values ? a->values + index : NULL; }

gchar *g_strdup(const gchar *s) { return s ? strdup(s) : NULL; }

gchar *g_strdup_printf(const gchar *fmt, ...)
{
    va_list ap, ap2;
    va_start(ap, fmt);
    va_copy(ap2, ap);
    int n = vsnprintf(NULL, 0, fmt, ap);
    va_end(ap);
    gchar *s = (gchar *)malloc((size_t)n + 1);
    vsnprintf(s, (size_t)n + 1, fmt, ap2);
    va_end(ap2);
    return s;
}

gchar *g_strconcat(const gchar *first, ...)
{
    std::string out;
    if (!first) return strdup("");
    out += first;
    va_list ap;
    va_start(ap, first);
    for (const gchar *s = va_arg(ap, const gchar *); s; s = va_arg(ap, const gchar *)) out += s;
    va_end(ap);
    return strdup(out.c_str());
}

gchar *g_strnfill(gsize length, gchar c)
{
    gchar *s = (gchar *)malloc(length + 1);
    memset(s, c, length);
    s[length] = 0;
    return s;
}

gchar *g_stpcpy(gchar *dest, const gchar *src) { return stpcpy(dest, src); }

gint g_strcmp0(const gchar *a, const gchar *b)
{
    if (!a) return -(a != b);
    if (!b) return a != b;
    return strcmp(a, b);
}

gchar **g_strsplit(const gchar *s, const gchar *delim, gint max_tokens)
{
    std::vector<std::string> parts;
    std::string str(s ? s : "");
    const size_t dl = strlen(delim);
    if (max_tokens < 1) max_tokens = INT_MAX;
    size_t pos = 0;
    if (!str.empty()) {
        while ((gint)parts.size() + 1 < max_tokens) {
            size_t hit = str.find(delim, pos);
            if (hit == std::string::npos) break;
            parts.push_back(str.substr(pos, hit - pos));
            pos = hit + dl;
        }
        parts.push_back(str.substr(pos));
    }
    gchar **v = (gchar **)calloc(parts.size() + 1, sizeof(gchar *));
    for (size_t i = 0; i < parts.size(); i++) v[i] = strdup(parts[i].c_str());
    return v;
}

void g_strfreev(gchar **v)
{
    if (!v) return;
    for (gchar **p = v; *p; p++) free(*p);
    free(v);
}

struct _GRegex {
    std::regex re;
};

GRegex *g_regex_new(const gchar *pattern, int, int, void *) { return new _GRegex{std::regex(pattern)}; }

gchar *g_regex_replace_literal(GRegex *re, const gchar *string, gssize len, gint start, const gchar *replacement,
                               int, void *)
{
    std::string s = len < 0 ? std::string(string) : std::string(string, (size_t)len);
    std::string head = s.substr(0, (size_t)start);
    std::string lit;  // "$" starts a back-reference in the ECMAScript format: double it
    for (const gchar *p = replacement; *p; p++) lit += *p == '$' ? "$$" : std::string(1, *p);
    std::string out = std::regex_replace(s.substr((size_t)start), re->re, lit);
    return strdup((head + out).c_str());
}

void g_regex_unref(GRegex *re) { delete re; }

guint g_str_hash(gconstpointer v)
{
    guint h = 5381;
    for (const unsigned char *p = (const unsigned char *)v; *p; p++) h = h * 33 + *p;
    return h;
}

gboolean g_str_equal(gconstpointer a, gconstpointer b) { return !strcmp((const char *)a, (const char *)b); }

struct _GHashTable {
    gboolean (*equal)(gconstpointer, gconstpointer);
    std::vector<std::pair<gpointer, gpointer>> items;
};

GHashTable *g_hash_table_new(guint (*)(gconstpointer), gboolean (*equal)(gconstpointer, gconstpointer))
{
    GHashTable *t = new _GHashTable;
    t->equal = equal;
    return t;
}

gboolean g_hash_table_insert(GHashTable *t, gpointer key, gpointer value)
{
    for (auto &kv : t->items)
        if (t->equal(kv.first, key)) {
            kv.second = value;
            return FALSE;
        }
    t->items.emplace_back(key, value);
    return TRUE;
}

gpointer g_hash_table_lookup(GHashTable *t, gconstpointer key)
{
    for (auto &kv : t->items)
        if (t->equal(kv.first, key)) return kv.second;
    return NULL;
}

void g_hash_table_destroy(GHashTable *t) { delete t; }

void g_log(const gchar *, int, const gchar *, ...) {}

void g_warning(const gchar *fmt, ...)
{
    va_list ap;
    va_start(ap, fmt);
    fprintf(stderr, "refshim warning: ");
    vfprintf(stderr, fmt, ap);
    fprintf(stderr, "\n");
    va_end(ap);
}

void g_set_error_literal(GError **err, int domain, int code, const char *message) { g_set_error(err, domain, code, "%s", message); }

void g_object_get(gpointer, const gchar *first, ...)
{
    va_list ap;
    va_start(ap, first);
    for (const gchar *name = first; name; name = va_arg(ap, const gchar *)) {
        if (!strcmp(name, "num_processed") || !strcmp(name, "num-processed")) {
            guint *out = va_arg(ap, guint *);
            *out = refshim_num_processed;
        } else {
            fprintf(stderr, "refshim: g_object_get of unknown property %s\n", name);
            abort();
        }
    }
    va_end(ap);
}

}  // extern "C"
