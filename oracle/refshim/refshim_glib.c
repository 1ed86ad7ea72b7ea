/* glib stand-in (declarations in oracle/refshim/glib.h): the GSList calls of
 * the reference's accelsearch, with glib's documented semantics.  Test
 * infrastructure only, written for this repository. */
#include <stdlib.h>

#include "glib.h"

GSList *g_slist_alloc(void) { return (GSList *) calloc(1, sizeof(GSList)); }

void g_slist_free_1(GSList *list) { free(list); }

void g_slist_free(GSList *list)
{
    while (list) {
        GSList *next = list->next;
        free(list);
        list = next;
    }
}

guint g_slist_length(GSList *list)
{
    guint n = 0;
    for (; list; list = list->next) n++;
    return n;
}

/* unlinks link_ from list (not freed; its next set to NULL) */
GSList *g_slist_remove_link(GSList *list, GSList *link_)
{
    GSList *prev = NULL, *cur = list;
    while (cur && cur != link_) {
        prev = cur;
        cur = cur->next;
    }
    if (cur) {
        if (prev) prev->next = cur->next;
        else list = cur->next;
        cur->next = NULL;
    }
    return list;
}

GSList *g_slist_prepend(GSList *list, gpointer data)
{
    GSList *n = g_slist_alloc();
    n->data = data;
    n->next = list;
    return n;
}

/* the next node is read before func runs, so func may free the current one */
void g_slist_foreach(GSList *list, GFunc func, gpointer user_data)
{
    while (list) {
        GSList *next = list->next;
        func(list->data, user_data);
        list = next;
    }
}

/* stable merge sort: on equal keys the node from the first run goes first */
static GSList *merge(GSList *a, GSList *b, GCompareFunc cmp)
{
    GSList head = {0}, *t = &head;
    while (a && b) {
        if (cmp(a->data, b->data) <= 0) {
            t->next = a;
            a = a->next;
        } else {
            t->next = b;
            b = b->next;
        }
        t = t->next;
    }
    t->next = a ? a : b;
    return head.next;
}

GSList *g_slist_sort(GSList *list, GCompareFunc compare_func)
{
    if (!list || !list->next) return list;
    GSList *slow = list, *fast = list->next;
    while (fast && fast->next) {
        slow = slow->next;
        fast = fast->next->next;
    }
    GSList *second = slow->next;
    slow->next = NULL;
    return merge(g_slist_sort(list, compare_func), g_slist_sort(second, compare_func),
                 compare_func);
}
