/* Stand-in for glib.h: the singly linked list subset that the reference's
 * accelsearch uses (GSList, include/accel.h and src/accel_utils.c),
 * implemented by oracle/refshim/refshim_glib.c with glib's documented
 * semantics (g_slist_sort is a stable merge sort).  Test infrastructure only. */
#ifndef REFSHIM_GLIB_H
#define REFSHIM_GLIB_H
typedef void *gpointer;
typedef const void *gconstpointer;
typedef int gint;
typedef unsigned int guint;
typedef gint gboolean;
#ifndef FALSE
#define FALSE (0)
#endif
#ifndef TRUE
#define TRUE (!FALSE)
#endif
typedef struct _GSList GSList;
struct _GSList {
    gpointer data;
    GSList *next;
};
typedef gint (*GCompareFunc)(gconstpointer a, gconstpointer b);
typedef void (*GFunc)(gpointer data, gpointer user_data);
GSList *g_slist_alloc(void);
void g_slist_free_1(GSList *list);
void g_slist_free(GSList *list);
guint g_slist_length(GSList *list);
GSList *g_slist_remove_link(GSList *list, GSList *link_);
GSList *g_slist_sort(GSList *list, GCompareFunc compare_func);
void g_slist_foreach(GSList *list, GFunc func, gpointer user_data);
GSList *g_slist_prepend(GSList *list, gpointer data);
#endif
