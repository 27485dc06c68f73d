/* Minimal ufo-core surface needed to compile the reference's task sources on a
 * machine without ufo-core, glib or OpenCL.  Types carry only what those
 * sources touch; the functions are implemented by ref_runtime.cpp and
 * ref_clc_jit.cpp, which run the tasks' OpenCL kernels (compiled as C++) on the
 * CPU.  Test infrastructure only. */
#ifndef REFSHIM_UFO_H
#define REFSHIM_UFO_H
#include <CL/cl.h>
#include <glib.h>
#ifdef __cplusplus
extern "C" {
#endif
/* every task struct is { UfoTaskNode parent_instance; <Task>Private *priv; } */
#define G_TYPE_INSTANCE_GET_PRIVATE(obj, type, ctype) (*(ctype **)((char *)(obj) + sizeof(UfoTaskNode)))
#define G_DEFINE_TYPE_WITH_CODE(TN, t_n, T_P, _C_)                \
    static void t_n##_init(TN *self);                             \
    static void t_n##_class_init(TN##Class *klass);               \
    static gpointer t_n##_parent_class = NULL;                    \
    GType t_n##_get_type(void) { return (GType)1; }

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
typedef enum {
    UFO_GPU_NODE_INFO_GLOBAL_MEM_SIZE,
    UFO_GPU_NODE_INFO_MAX_MEM_ALLOC_SIZE,
    UFO_GPU_NODE_INFO_LOCAL_MEM_SIZE,
    UFO_GPU_NODE_INFO_MAX_WORK_GROUP_SIZE,
    UFO_GPU_NODE_INFO_NAME
} UfoGpuNodeInfo;
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
GValue *ufo_gpu_node_get_info(UfoGpuNode *node, UfoGpuNodeInfo info);
cl_context ufo_resources_get_context(UfoResources *res);
cl_kernel ufo_resources_get_kernel(UfoResources *res, const char *file, const char *name, const char *opts,
                                   GError **err);
gchar *ufo_resources_get_kernel_source(UfoResources *res, const gchar *filename, GError **err);
cl_kernel ufo_resources_get_kernel_from_source(UfoResources *res, const gchar *source, const gchar *name,
                                               const gchar *opts, GError **err);
void ufo_buffer_get_requisition(UfoBuffer *buf, UfoRequisition *req);
cl_mem ufo_buffer_get_device_array(UfoBuffer *buf, cl_command_queue q);
cl_mem ufo_buffer_get_device_image(UfoBuffer *buf, cl_command_queue q);
gfloat *ufo_buffer_get_host_array(UfoBuffer *buf, cl_command_queue q);
gfloat ufo_buffer_min(UfoBuffer *buf, cl_command_queue q);
gfloat ufo_buffer_max(UfoBuffer *buf, cl_command_queue q);
void ufo_profiler_call(UfoProfiler *p, cl_command_queue q, cl_kernel k, guint ndims, const gsize *global,
                       const gsize *local);
void ufo_profiler_call_blocking(UfoProfiler *p, cl_command_queue q, cl_kernel k, guint ndims, const gsize *global,
                                const gsize *local);
#ifdef __cplusplus
}
#endif
#endif
