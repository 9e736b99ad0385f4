/*
 * json.h - TEST INFRASTRUCTURE ONLY: a stand-in for libjson's event parser, which the
 * reference's json_parser.cc includes as <json.h> and links from the system (the library
 * is not part of the reference tree and its version is not pinned there).
 *
 * Only the interface json_parser.cc uses is offered: json_parser_init / _string / _is_done /
 * _free and the event codes.  Events carry the token's text, NUL-terminated: a key or string
 * unescaped, a number as written; true, false and null carry none.  The stand-in collects
 * the input and parses it when json_parser_is_done is called, delivering the same events
 * in the same order as a streaming parser would.  Implemented in ../json_shim.c.
 */
#ifndef RZK_JSON_SHIM_H_
#define RZK_JSON_SHIM_H_

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum {
    JSON_NONE = 0,
    JSON_ARRAY_BEGIN,
    JSON_OBJECT_BEGIN,
    JSON_ARRAY_END,
    JSON_OBJECT_END,
    JSON_INT,
    JSON_FLOAT,
    JSON_STRING,
    JSON_KEY,
    JSON_TRUE,
    JSON_FALSE,
    JSON_NULL,
    JSON_BSTRING
};

typedef int (*json_parser_callback)(void *userdata, int type, const char *data, uint32_t length);

typedef struct {
    uint32_t buffer_initial_size;
    uint32_t max_nesting;
    uint32_t max_data;
    int allow_c_comments;
    int allow_yaml_comments;
    void *(*user_calloc)(size_t nmemb, size_t size);
    void *(*user_realloc)(void *ptr, size_t size);
} json_config;

typedef struct json_parser {
    json_parser_callback callback;
    void *userdata;
    char *text;
    size_t len, cap;
} json_parser;

int json_parser_init(json_parser *parser, json_config *cfg, json_parser_callback callback, void *userdata);
int json_parser_free(json_parser *parser);
/* appends the input; returns 0 and *processed = length */
int json_parser_string(json_parser *parser, const char *string, uint32_t length, uint32_t *processed);
/* parses everything appended: 1 for one complete, valid document, 0 otherwise */
int json_parser_is_done(json_parser *parser);

#ifdef __cplusplus
}
#endif

#endif
