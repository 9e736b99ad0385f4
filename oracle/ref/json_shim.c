/*
 * json_shim.c - TEST INFRASTRUCTURE ONLY: the libjson stand-in declared in shim/json.h, a
 * recursive-descent reader of RFC 8259 text that delivers libjson's events (begin / end of
 * objects and arrays, keys, strings, integers, reals, true, false, null).  A number without
 * a fraction or exponent is JSON_INT, any other JSON_FLOAT.
 */
#include <stdlib.h>
#include <string.h>

#include "shim/json.h"

typedef struct {
    const char *p, *end;
    json_parser *jp;
    char *tok;
    size_t tok_len, tok_cap;
    int ok;
} Reader;

static void tok_reset(Reader *r) { r->tok_len = 0; }

static void tok_put(Reader *r, char c) {
    if (r->tok_len + 2 > r->tok_cap) {
        r->tok_cap = r->tok_cap ? 2 * r->tok_cap : 256;
        r->tok = (char *)realloc(r->tok, r->tok_cap);
    }
    r->tok[r->tok_len++] = c;
    r->tok[r->tok_len] = 0;
}

static void emit(Reader *r, int type, int with_text) {
    if (!r->ok) return;
    if (with_text) {
        if (!r->tok) tok_put(r, 0), r->tok_len = 0;
        r->tok[r->tok_len] = 0;
        r->jp->callback(r->jp->userdata, type, r->tok, (uint32_t)r->tok_len);
    } else {
        r->jp->callback(r->jp->userdata, type, NULL, 0);
    }
}

static void ws(Reader *r) {
    while (r->p < r->end && (*r->p == ' ' || *r->p == '\t' || *r->p == '\n' || *r->p == '\r')) r->p++;
}

static int hex4(Reader *r, unsigned *out) {
    unsigned v = 0;
    if (r->end - r->p < 4) return 0;
    for (int i = 0; i < 4; ++i) {
        char c = *r->p++;
        v <<= 4;
        if (c >= '0' && c <= '9') v |= (unsigned)(c - '0');
        else if (c >= 'a' && c <= 'f') v |= (unsigned)(c - 'a' + 10);
        else if (c >= 'A' && c <= 'F') v |= (unsigned)(c - 'A' + 10);
        else return 0;
    }
    *out = v;
    return 1;
}

static void put_utf8(Reader *r, unsigned cp) {
    if (cp < 0x80) {
        tok_put(r, (char)cp);
    } else if (cp < 0x800) {
        tok_put(r, (char)(0xc0 | (cp >> 6)));
        tok_put(r, (char)(0x80 | (cp & 0x3f)));
    } else if (cp < 0x10000) {
        tok_put(r, (char)(0xe0 | (cp >> 12)));
        tok_put(r, (char)(0x80 | ((cp >> 6) & 0x3f)));
        tok_put(r, (char)(0x80 | (cp & 0x3f)));
    } else {
        tok_put(r, (char)(0xf0 | (cp >> 18)));
        tok_put(r, (char)(0x80 | ((cp >> 12) & 0x3f)));
        tok_put(r, (char)(0x80 | ((cp >> 6) & 0x3f)));
        tok_put(r, (char)(0x80 | (cp & 0x3f)));
    }
}

/* a string into the token buffer; 0 on a syntax error */
static int string(Reader *r) {
    tok_reset(r);
    tok_put(r, 0);
    r->tok_len = 0;
    if (r->p >= r->end || *r->p != '"') return 0;
    r->p++;
    for (;;) {
        if (r->p >= r->end) return 0;
        unsigned char c = (unsigned char)*r->p++;
        if (c == '"') return 1;
        if (c < 0x20) return 0;
        if (c != '\\') { tok_put(r, (char)c); continue; }
        if (r->p >= r->end) return 0;
        char e = *r->p++;
        unsigned cp, lo;
        switch (e) {
        case '"': tok_put(r, '"'); break;
        case '\\': tok_put(r, '\\'); break;
        case '/': tok_put(r, '/'); break;
        case 'b': tok_put(r, '\b'); break;
        case 'f': tok_put(r, '\f'); break;
        case 'n': tok_put(r, '\n'); break;
        case 'r': tok_put(r, '\r'); break;
        case 't': tok_put(r, '\t'); break;
        case 'u':
            if (!hex4(r, &cp)) return 0;
            if (cp >= 0xd800 && cp < 0xdc00) {
                if (r->end - r->p < 6 || r->p[0] != '\\' || r->p[1] != 'u') return 0;
                r->p += 2;
                if (!hex4(r, &lo) || lo < 0xdc00 || lo >= 0xe000) return 0;
                cp = 0x10000 + ((cp - 0xd800) << 10) + (lo - 0xdc00);
            } else if (cp >= 0xdc00 && cp < 0xe000) {
                return 0;
            }
            put_utf8(r, cp);
            break;
        default: return 0;
        }
    }
}

static int digits(Reader *r) {
    if (r->p >= r->end || *r->p < '0' || *r->p > '9') return 0;
    while (r->p < r->end && *r->p >= '0' && *r->p <= '9') tok_put(r, *r->p++);
    return 1;
}

static int number(Reader *r) {
    int real = 0;
    tok_reset(r);
    if (r->p < r->end && *r->p == '-') tok_put(r, *r->p++);
    if (r->p >= r->end) return 0;
    if (*r->p == '0') tok_put(r, *r->p++);
    else if (!digits(r)) return 0;
    if (r->p < r->end && *r->p == '.') {
        real = 1;
        tok_put(r, *r->p++);
        if (!digits(r)) return 0;
    }
    if (r->p < r->end && (*r->p == 'e' || *r->p == 'E')) {
        real = 1;
        tok_put(r, *r->p++);
        if (r->p < r->end && (*r->p == '+' || *r->p == '-')) tok_put(r, *r->p++);
        if (!digits(r)) return 0;
    }
    emit(r, real ? JSON_FLOAT : JSON_INT, 1);
    return 1;
}

static int word(Reader *r, const char *w) {
    size_t n = strlen(w);
    if ((size_t)(r->end - r->p) < n || strncmp(r->p, w, n) != 0) return 0;
    r->p += n;
    return 1;
}

static int value(Reader *r, int depth) {
    ws(r);
    if (r->p >= r->end || depth > 512) return 0;
    char c = *r->p;
    if (c == '{') {
        r->p++;
        emit(r, JSON_OBJECT_BEGIN, 0);
        ws(r);
        if (r->p < r->end && *r->p == '}') { r->p++; emit(r, JSON_OBJECT_END, 0); return 1; }
        for (;;) {
            ws(r);
            if (!string(r)) return 0;
            emit(r, JSON_KEY, 1);
            ws(r);
            if (r->p >= r->end || *r->p != ':') return 0;
            r->p++;
            if (!value(r, depth + 1)) return 0;
            ws(r);
            if (r->p < r->end && *r->p == ',') { r->p++; continue; }
            if (r->p < r->end && *r->p == '}') { r->p++; emit(r, JSON_OBJECT_END, 0); return 1; }
            return 0;
        }
    }
    if (c == '[') {
        r->p++;
        emit(r, JSON_ARRAY_BEGIN, 0);
        ws(r);
        if (r->p < r->end && *r->p == ']') { r->p++; emit(r, JSON_ARRAY_END, 0); return 1; }
        for (;;) {
            if (!value(r, depth + 1)) return 0;
            ws(r);
            if (r->p < r->end && *r->p == ',') { r->p++; continue; }
            if (r->p < r->end && *r->p == ']') { r->p++; emit(r, JSON_ARRAY_END, 0); return 1; }
            return 0;
        }
    }
    if (c == '"') {
        if (!string(r)) return 0;
        emit(r, JSON_STRING, 1);
        return 1;
    }
    if (word(r, "true")) { emit(r, JSON_TRUE, 0); return 1; }
    if (word(r, "false")) { emit(r, JSON_FALSE, 0); return 1; }
    if (word(r, "null")) { emit(r, JSON_NULL, 0); return 1; }
    return number(r);
}

int json_parser_init(json_parser *parser, json_config *cfg, json_parser_callback callback, void *userdata) {
    (void)cfg;
    memset(parser, 0, sizeof(*parser));
    parser->callback = callback;
    parser->userdata = userdata;
    return 0;
}

int json_parser_free(json_parser *parser) {
    free(parser->text);
    parser->text = NULL;
    parser->len = parser->cap = 0;
    return 0;
}

int json_parser_string(json_parser *parser, const char *string_in, uint32_t length, uint32_t *processed) {
    if (parser->len + length + 1 > parser->cap) {
        size_t cap = parser->cap ? parser->cap : 4096;
        while (cap < parser->len + length + 1) cap *= 2;
        parser->text = (char *)realloc(parser->text, cap);
        parser->cap = cap;
    }
    memcpy(parser->text + parser->len, string_in, length);
    parser->len += length;
    if (processed) *processed = length;
    return 0;
}

int json_parser_is_done(json_parser *parser) {
    Reader r;
    memset(&r, 0, sizeof(r));
    r.p = parser->text;
    r.end = parser->text + parser->len;
    r.jp = parser;
    r.ok = 1;
    int done = parser->len > 0 && value(&r, 0);
    if (done) {
        ws(&r);
        done = r.p == r.end;
    }
    free(r.tok);
    return done;
}
