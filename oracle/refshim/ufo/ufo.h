/* Minimal GLib / GObject / ufo-core surface needed to compile the reference's
 * `filter` and `backproject` task sources on a machine without ufo-core, glib or
 * OpenCL.  Types carry only what those sources touch; the functions are
 * implemented by ref_runtime.cpp, which runs the tasks' OpenCL kernels (compiled
 * as C++) on the CPU.  Test infrastructure only. */
#ifndef REFSHIM_UFO_H
#define REFSHIM_UFO_H
#include <CL/cl.h>
#include <float.h>
#include <limits.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef __cplusplus
extern "C" {
#endif
typedef float gfloat;
typedef double gdouble;
typedef int gint;
typedef unsigned int guint;
typedef int gboolean;
typedef size_t gsize;
typedef void *gpointer;
typedef char gchar;
typedef unsigned long GType;
#define TRUE 1
#define FALSE 0
#define G_PI 3.1415926535897932384626433832795028841971693993751
#define G_MAXFLOAT FLT_MAX
#define G_MAXDOUBLE DBL_MAX
#define G_MAXUINT UINT_MAX
#define G_BEGIN_DECLS
#define G_END_DECLS
typedef struct { int domain, code; char message[512]; } GError;
typedef struct { union { int i; unsigned u; float f; double d; } data; } GValue;
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
#define g_enum_register_static(name, values) ((GType)(values != NULL))
#define g_object_class_install_property(oclass, id, pspec) ((void)(oclass), (void)(id), (void)(pspec))
#define g_type_class_add_private(klass, size) ((void)(klass), (void)(size))
#define G_OBJECT_WARN_INVALID_PROPERTY_ID(obj, id, pspec) ((void)(obj), (void)(id), (void)(pspec))
#define g_value_get_enum(gv) ((gv)->data.i)
#define g_value_set_enum(gv, x) ((gv)->data.i = (x))
#define g_value_get_float(gv) ((gv)->data.f)
#define g_value_set_float(gv, x) ((gv)->data.f = (x))
#define g_value_get_double(gv) ((gv)->data.d)
#define g_value_set_double(gv, x) ((gv)->data.d = (x))
#define g_value_get_uint(gv) ((gv)->data.u)
#define g_value_set_uint(gv, x) ((gv)->data.u = (x))
#define g_return_val_if_fail(expr, val) do { if (!(expr)) return (val); } while (0)
#define g_malloc0(n) calloc(1, (n))
#define g_realloc(p, n) realloc((p), (n))
#define g_free(p) free(p)
void g_set_error(GError **err, int domain, int code, const char *fmt, ...);
void *g_object_new(GType type, ...);
#define G_OBJECT_CLASS(k) ((GObjectClass *)(k))
#define G_TYPE_CHECK_INSTANCE_CAST(obj, type, ctype) ((ctype *)(obj))
#define G_TYPE_CHECK_INSTANCE_TYPE(obj, type) ((obj) != NULL)
#define G_TYPE_CHECK_CLASS_CAST(k, type, ctype) ((ctype *)(k))
#define G_TYPE_CHECK_CLASS_TYPE(k, type) ((k) != NULL)
#define G_TYPE_INSTANCE_GET_CLASS(obj, type, ctype) ((ctype *)NULL)
/* every task struct is { UfoTaskNode parent_instance; <Task>Private *priv; } */
#define G_TYPE_INSTANCE_GET_PRIVATE(obj, type, ctype) (*(ctype **)((char *)(obj) + sizeof(UfoTaskNode)))
#define G_IMPLEMENT_INTERFACE(iface_type, init)
#define G_DEFINE_TYPE_WITH_CODE(TN, t_n, T_P, _C_)                \
    static void t_n##_init(TN *self);                             \
    static void t_n##_class_init(TN##Class *klass);               \
    static gpointer t_n##_parent_class = NULL;                    \
    GType t_n##_get_type(void) { return (GType)1; }

/* ufo-core */
typedef struct { void *dummy; } UfoNode;
typedef struct { GObjectClass parent; gboolean (*equal)(UfoNode *, UfoNode *); } UfoNodeClass;
typedef struct { void *dummy; } UfoTaskNode;
typedef struct { UfoNodeClass parent; } UfoTaskNodeClass;
typedef struct UfoTask UfoTask;
typedef struct { void *dummy; } UfoResources;
typedef struct { void *dummy; } UfoGpuNode;
typedef struct { void *dummy; } UfoProfiler;
typedef struct { guint n_dims; gsize dims[16]; } UfoRequisition;
typedef struct UfoBuffer UfoBuffer;
typedef enum { UFO_TASK_MODE_PROCESSOR = 1, UFO_TASK_MODE_GPU = 1 << 4, UFO_TASK_MODE_REDUCTOR = 2 } UfoTaskMode;
typedef struct {
    void (*setup)(UfoTask *, UfoResources *, GError **);
    void (*get_requisition)(UfoTask *, UfoBuffer **, UfoRequisition *, GError **);
    guint (*get_num_inputs)(UfoTask *);
    guint (*get_num_dimensions)(UfoTask *, guint);
    UfoTaskMode (*get_mode)(UfoTask *);
    gboolean (*process)(UfoTask *, UfoBuffer **, UfoBuffer *, UfoRequisition *);
    gboolean (*generate)(UfoTask *, UfoBuffer *, UfoRequisition *);
} UfoTaskIface;
#define UFO_TYPE_TASK_NODE ((GType)1)
#define UFO_TYPE_TASK ((GType)2)
#define UFO_TASK_ERROR 1
#define UFO_TASK_ERROR_SETUP 1
#define UFO_TASK_ERROR_GET_REQUISITION 2
#define UFO_NODE(obj) ((UfoNode *)(obj))
#define UFO_NODE_CLASS(k) ((UfoNodeClass *)(k))
#define UFO_TASK_NODE(obj) ((UfoTaskNode *)(obj))
#define UFO_GPU_NODE(obj) ((UfoGpuNode *)(obj))
#define UFO_RESOURCES_CHECK_CLERR(e) ((void)(e))
#define UFO_RESOURCES_CHECK_SET_AND_RETURN(e, err) ((void)(e))
UfoGpuNode *ufo_task_node_get_proc_node(UfoTaskNode *node);
UfoProfiler *ufo_task_node_get_profiler(UfoTaskNode *node);
cl_command_queue ufo_gpu_node_get_cmd_queue(UfoGpuNode *node);
cl_context ufo_resources_get_context(UfoResources *res);
cl_kernel ufo_resources_get_kernel(UfoResources *res, const char *file, const char *name, const char *opts,
                                   GError **err);
void ufo_buffer_get_requisition(UfoBuffer *buf, UfoRequisition *req);
cl_mem ufo_buffer_get_device_array(UfoBuffer *buf, cl_command_queue q);
cl_mem ufo_buffer_get_device_image(UfoBuffer *buf, cl_command_queue q);
void ufo_profiler_call(UfoProfiler *p, cl_command_queue q, cl_kernel k, guint ndims, const gsize *global,
                       const gsize *local);
#ifdef __cplusplus
}
#endif
#endif
