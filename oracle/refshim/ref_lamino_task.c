/* Drives the reference's own `lamino-backproject` task
 * (src/ufo-lamino-backproject-task.c with src/lamino-roi.c, compiled in this
 * translation unit against the CPU shims) the way ufo-core does: properties
 * through the task's set_property, setup, get_requisition, process once per
 * projection into the volume, then generate.  Its kernels are the ones
 * src/kernels/tools/make_burst_kernels.py writes from
 * src/kernels/templates/{z,center,lamino,roll}_template.in at build time
 * (src/kernels/meson.build:59-83; oracle/reference.py runs the script), compiled
 * for the CPU by ref_clc_jit.cpp.  BURST is the build option's default
 * (meson_options.txt: lamino_backproject_burst_mode = 16).  Test
 * infrastructure only. */
#define BURST 16
#include "ufo-lamino-backproject-task.c"
#include "lamino-roi.c"
#include "refshim_internal.h"

typedef struct {
    UfoLaminoBackprojectTask task;
    UfoLaminoBackprojectTaskPrivate *priv;
} RefLamino;

static const struct {
    const char *name;
    guint id;
    GType type; /* element type of value arrays, or the scalar's type */
} lamino_props[] = {
    {"x-region", PROP_X_REGION, G_TYPE_INT},
    {"y-region", PROP_Y_REGION, G_TYPE_INT},
    {"z", PROP_Z, G_TYPE_FLOAT},
    {"region", PROP_REGION, G_TYPE_FLOAT},
    {"projection-offset", PROP_PROJECTION_OFFSET, G_TYPE_INT},
    {"center", PROP_CENTER, G_TYPE_FLOAT},
    {"num-projections", PROP_NUM_PROJECTIONS, G_TYPE_UINT},
    {"overall-angle", PROP_OVERALL_ANGLE, G_TYPE_FLOAT},
    {"tomo-angle", PROP_TOMO_ANGLE, G_TYPE_FLOAT},
    {"lamino-angle", PROP_LAMINO_ANGLE, G_TYPE_FLOAT},
    {"parameter", PROP_PARAMETER, G_TYPE_ENUM},
    {"roll-angle", PROP_ROLL_ANGLE, G_TYPE_FLOAT},
    {"addressing-mode", PROP_ADDRESSING_MODE, G_TYPE_ENUM},
};

void *ref_lamino_new(void)
{
    RefLamino *g = (RefLamino *)calloc(1, sizeof(RefLamino));
    g->priv = (UfoLaminoBackprojectTaskPrivate *)calloc(1, sizeof(UfoLaminoBackprojectTaskPrivate));
    g->task.priv = g->priv;
    ufo_lamino_backproject_task_init(&g->task);
    return g;
}

/* Set one property by its reference name: value arrays (regions, center,
 * projection offset) from n doubles converted to the task's element type,
 * scalars from values[0], enumerations by their value nick.  Returns 0, or -1
 * for an unknown name or nick. */
int ref_lamino_set(void *handle, const char *name, const double *values, unsigned n, const char *nick)
{
    RefLamino *g = (RefLamino *)handle;
    GValue v = G_VALUE_INIT;
    unsigned i, k;
    for (k = 0; k < sizeof lamino_props / sizeof lamino_props[0]; k++)
        if (!strcmp(lamino_props[k].name, name)) break;
    if (k == sizeof lamino_props / sizeof lamino_props[0]) return -1;
    switch (lamino_props[k].id) {
        case PROP_X_REGION:
        case PROP_Y_REGION:
        case PROP_REGION:
        case PROP_PROJECTION_OFFSET:
        case PROP_CENTER: {
            GValueArray *a = g_value_array_new(n);
            GValue e = G_VALUE_INIT;
            g_value_init(&e, lamino_props[k].type);
            for (i = 0; i < n; i++) {
                if (lamino_props[k].type == G_TYPE_INT)
                    g_value_set_int(&e, (int)values[i]);
                else
                    g_value_set_float(&e, (float)values[i]);
                g_value_array_append(a, &e);
            }
            g_value_init(&v, G_TYPE_VALUE_ARRAY);
            g_value_set_boxed(&v, a);
            ufo_lamino_backproject_task_set_property((GObject *)&g->task, lamino_props[k].id, &v, NULL);
            g_value_array_free(a);
            return 0;
        }
        case PROP_PARAMETER:
        case PROP_ADDRESSING_MODE: {
            const GEnumValue *t = lamino_props[k].id == PROP_PARAMETER ? parameter_values : addressing_values;
            for (; t->value_nick; t++)
                if (nick && !strcmp(t->value_nick, nick)) break;
            if (!t->value_nick) return -1;
            g_value_init(&v, G_TYPE_ENUM);
            g_value_set_enum(&v, t->value);
            break;
        }
        case PROP_NUM_PROJECTIONS:
            g_value_init(&v, G_TYPE_UINT);
            g_value_set_uint(&v, (guint)values[0]);
            break;
        default:
            g_value_init(&v, G_TYPE_FLOAT);
            g_value_set_float(&v, (float)values[0]);
            break;
    }
    ufo_lamino_backproject_task_set_property((GObject *)&g->task, lamino_props[k].id, &v, NULL);
    return 0;
}

/* Run the task over `count` projections of width x height floats into `out`
 * (dims gets x, y, z of the requisition; nothing is computed when out is NULL
 * or too small).  Returns 0, or -1 with the task's GError message in err. */
int ref_lamino_run(void *handle, const float *proj, unsigned width, unsigned height, unsigned count, float *out,
                   size_t out_floats, unsigned *dims, char *err, int errlen)
{
    RefLamino *g = (RefLamino *)handle;
    UfoTask *task = (UfoTask *)&g->task;
    GError *e = NULL;
    UfoBuffer in, ob;
    UfoBuffer *inputs[1] = {&in};
    UfoRequisition req;
    unsigned i;

    memset(&req, 0, sizeof req);
    ufo_lamino_backproject_task_setup(task, NULL, &e);
    if (e) {
        snprintf(err, errlen, "%s", e->message);
        free(e);
        return -1;
    }
    refshim_buffer_init(&in, (float *)proj, 2, width, height, 1);
    ufo_lamino_backproject_task_get_requisition(task, inputs, &req, &e);
    dims[0] = (unsigned)req.dims[0];
    dims[1] = (unsigned)req.dims[1];
    dims[2] = (unsigned)req.dims[2];
    if (!out || (size_t)dims[0] * dims[1] * dims[2] > out_floats) return 0;
    refshim_buffer_init(&ob, out, 3, dims[0], dims[1], dims[2]);
    for (i = 0; i < count; i++) {
        refshim_num_processed = i;
        refshim_buffer_init(&in, (float *)proj + (size_t)i * width * height, 2, width, height, 1);
        ufo_lamino_backproject_task_process(task, inputs, &ob, &req);
    }
    refshim_num_processed = count;
    ufo_lamino_backproject_task_generate(task, &ob, &req);
    return 0;
}
