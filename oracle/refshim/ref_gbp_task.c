/* Drives the reference's own `general-backproject` task
 * (src/ufo-general-backproject-task.c, compiled in this translation unit
 * against the CPU shims, with src/common/ufo-scarray.c, ufo-ctgeometry.c and
 * ufo-conebeam.c beside it) the way ufo-core does: properties through the
 * task's set_property, setup, then get_requisition + process once per
 * projection with the node's "num_processed" count, then generate once per
 * slice.  The kernel the task generates (make_kernel) is compiled for the CPU
 * by ref_clc_jit.cpp.  Test infrastructure only. */
#include "ufo-general-backproject-task.c"
#include "refshim_internal.h"

typedef struct {
    UfoGeneralBackprojectTask task;
    UfoGeneralBackprojectTaskPrivate *priv;
} RefGbp;

static const struct {
    const char *name;
    guint id;
} gbp_props[] = {
    {"burst", PROP_BURST},
    {"parameter", PROP_PARAMETER},
    {"z", PROP_Z},
    {"region", PROP_REGION},
    {"x-region", PROP_REGION_X},
    {"y-region", PROP_REGION_Y},
    {"center-position-x", PROP_CENTER_POSITION_X},
    {"center-position-z", PROP_CENTER_POSITION_Z},
    {"source-position-x", PROP_SOURCE_POSITION_X},
    {"source-position-y", PROP_SOURCE_POSITION_Y},
    {"source-position-z", PROP_SOURCE_POSITION_Z},
    {"detector-position-x", PROP_DETECTOR_POSITION_X},
    {"detector-position-y", PROP_DETECTOR_POSITION_Y},
    {"detector-position-z", PROP_DETECTOR_POSITION_Z},
    {"detector-angle-x", PROP_DETECTOR_ANGLE_X},
    {"detector-angle-y", PROP_DETECTOR_ANGLE_Y},
    {"detector-angle-z", PROP_DETECTOR_ANGLE_Z},
    {"axis-angle-x", PROP_AXIS_ANGLE_X},
    {"axis-angle-y", PROP_AXIS_ANGLE_Y},
    {"axis-angle-z", PROP_AXIS_ANGLE_Z},
    {"volume-angle-x", PROP_VOLUME_ANGLE_X},
    {"volume-angle-y", PROP_VOLUME_ANGLE_Y},
    {"volume-angle-z", PROP_VOLUME_ANGLE_Z},
    {"num-projections", PROP_NUM_PROJECTIONS},
    {"compute-type", PROP_COMPUTE_TYPE},
    {"result-type", PROP_RESULT_TYPE},
    {"store-type", PROP_STORE_TYPE},
    {"overall-angle", PROP_OVERALL_ANGLE},
    {"addressing-mode", PROP_ADDRESSING_MODE},
    {"gray-map-min", PROP_GRAY_MAP_MIN},
    {"gray-map-max", PROP_GRAY_MAP_MAX},
};

static int nick_value(const GEnumValue *table, const char *nick)
{
    for (; table->value_nick; table++)
        if (!strcmp(table->value_nick, nick)) return table->value;
    return -1;
}

void *ref_gbp_new(void)
{
    RefGbp *g = (RefGbp *)calloc(1, sizeof(RefGbp));
    g->priv = (UfoGeneralBackprojectTaskPrivate *)calloc(1, sizeof(UfoGeneralBackprojectTaskPrivate));
    g->task.priv = g->priv;
    ufo_general_backproject_task_init(&g->task);
    return g;
}

/* Set one property by its reference name.  Enumerations take `nick` (the
 * reference's value nicks), uint/double properties values[0], and the
 * UfoScarray properties a GValueArray of the n doubles.  Returns 0, or -1 for
 * an unknown name or nick. */
int ref_gbp_set(void *handle, const char *name, const double *values, unsigned n, const char *nick)
{
    RefGbp *g = (RefGbp *)handle;
    GValue v = G_VALUE_INIT;
    guint id = 0, i;
    for (i = 0; i < sizeof gbp_props / sizeof gbp_props[0]; i++)
        if (!strcmp(gbp_props[i].name, name)) id = gbp_props[i].id;
    if (!id) return -1;
    switch (id) {
        case PROP_PARAMETER:
        case PROP_COMPUTE_TYPE:
        case PROP_RESULT_TYPE:
        case PROP_STORE_TYPE:
        case PROP_ADDRESSING_MODE: {
            const GEnumValue *table = id == PROP_PARAMETER      ? parameter_values
                                      : id == PROP_COMPUTE_TYPE ? compute_type_values
                                      : id == PROP_RESULT_TYPE  ? ft_values
                                      : id == PROP_STORE_TYPE   ? st_values
                                                                : addressing_values;
            int e = nick ? nick_value(table, nick) : -1;
            if (e < 0) return -1;
            g_value_init(&v, G_TYPE_ENUM);
            g_value_set_enum(&v, e);
            break;
        }
        case PROP_BURST:
        case PROP_NUM_PROJECTIONS:
            g_value_init(&v, G_TYPE_UINT);
            g_value_set_uint(&v, (guint)values[0]);
            break;
        case PROP_Z:
        case PROP_OVERALL_ANGLE:
        case PROP_GRAY_MAP_MIN:
        case PROP_GRAY_MAP_MAX:
            g_value_init(&v, G_TYPE_DOUBLE);
            g_value_set_double(&v, values[0]);
            break;
        default: {
            GValueArray *a = g_value_array_new(n);
            GValue d = G_VALUE_INIT;
            g_value_init(&d, G_TYPE_DOUBLE);
            for (i = 0; i < n; i++) {
                g_value_set_double(&d, values[i]);
                g_value_array_append(a, &d);
            }
            g_value_init(&v, G_TYPE_VALUE_ARRAY);
            g_value_set_boxed(&v, a);
            ufo_general_backproject_task_set_property((GObject *)&g->task, id, &v, NULL);
            g_value_array_free(a);
            return 0;
        }
    }
    ufo_general_backproject_task_set_property((GObject *)&g->task, id, &v, NULL);
    return 0;
}

static int fail(GError *e, char *err, int errlen)
{
    snprintf(err, errlen, "%s", e->message);
    free(e);
    return -1;
}

/* Run the task over `count` projections of width x height floats.  dims gets
 * (slice width, slice height, slices, bytes per voxel); the volume is written
 * to `out` when it fits in out_bytes.  Returns the number of slices generated,
 * or -1 with the task's GError message in err. */
int ref_gbp_run(void *handle, const float *proj, unsigned width, unsigned height, unsigned count, void *out,
                size_t out_bytes, unsigned *dims, char *err, int errlen)
{
    RefGbp *g = (RefGbp *)handle;
    UfoTask *task = (UfoTask *)&g->task;
    GError *e = NULL;
    UfoBuffer in, ob;
    UfoBuffer *inputs[1] = {&in};
    UfoRequisition req;
    size_t slice_bytes;
    unsigned i;
    int s;

    memset(&req, 0, sizeof req);
    ufo_general_backproject_task_setup(task, NULL, &e);
    if (e) return fail(e, err, errlen);
    for (i = 0; i < count; i++) {
        refshim_num_processed = i;
        refshim_buffer_init(&in, (float *)proj + (size_t)i * width * height, 2, width, height, 1);
        ufo_general_backproject_task_get_requisition(task, inputs, &req, &e);
        if (e) return fail(e, err, errlen);
        ufo_general_backproject_task_process(task, inputs, NULL, &req);
    }
    refshim_num_processed = count;
    dims[0] = (unsigned)req.dims[0];
    dims[1] = (unsigned)req.dims[1];
    dims[2] = g->priv->num_slices;
    dims[3] = (unsigned)get_type_size(g->priv->store_type);
    slice_bytes = (size_t)dims[0] * dims[1] * dims[3];
    if (!out || slice_bytes * dims[2] > out_bytes) return 0;
    for (s = 0;; s++) {
        refshim_buffer_init_bytes(&ob, (char *)out + (size_t)s * slice_bytes, slice_bytes, 2, dims[0], dims[1], 1);
        if (!ufo_general_backproject_task_generate(task, &ob, &req)) break;
    }
    return s;
}
