/* json.c -- the small JSON reader the bundle loader needs for index.json,
 * index.pq.json and index.pqresN.json (RFC 8259: objects, arrays, strings
 * with escapes, numbers, true / false / null). */
#include "json.h"

#include <stdio.h>
#include <stdlib.h>
#include <string.h>

typedef struct {
    const char* p;
    const char* end;
    char* err;
    size_t errlen;
    int depth;
} Parser;

static int fail(Parser* ps, const char* what) {
    if (ps->err && ps->errlen) snprintf(ps->err, ps->errlen, "JSON: %s", what);
    return -1;
}

static void skip_ws(Parser* ps) {
    while (ps->p < ps->end && (*ps->p == ' ' || *ps->p == '\t' || *ps->p == '\n' || *ps->p == '\r')) ++ps->p;
}

static int put_utf8(char** buf, size_t* len, size_t* cap, uint32_t cp) {
    char tmp[4];
    int n;
    if (cp < 0x80) { tmp[0] = (char)cp; n = 1; }
    else if (cp < 0x800) { tmp[0] = (char)(0xC0 | (cp >> 6)); tmp[1] = (char)(0x80 | (cp & 63)); n = 2; }
    else if (cp < 0x10000) {
        tmp[0] = (char)(0xE0 | (cp >> 12)); tmp[1] = (char)(0x80 | ((cp >> 6) & 63)); tmp[2] = (char)(0x80 | (cp & 63));
        n = 3;
    } else {
        tmp[0] = (char)(0xF0 | (cp >> 18)); tmp[1] = (char)(0x80 | ((cp >> 12) & 63));
        tmp[2] = (char)(0x80 | ((cp >> 6) & 63)); tmp[3] = (char)(0x80 | (cp & 63));
        n = 4;
    }
    if (*len + n + 1 > *cap) {
        size_t c = *cap ? *cap * 2 : 32;
        while (c < *len + n + 1) c *= 2;
        char* nb = (char*)realloc(*buf, c);
        if (!nb) return -1;
        *buf = nb;
        *cap = c;
    }
    memcpy(*buf + *len, tmp, n);
    *len += n;
    (*buf)[*len] = '\0';
    return 0;
}

static int hex4(Parser* ps, uint32_t* out) {
    if (ps->end - ps->p < 4) return -1;
    uint32_t v = 0;
    for (int i = 0; i < 4; ++i) {
        const char c = ps->p[i];
        v <<= 4;
        if (c >= '0' && c <= '9') v |= (uint32_t)(c - '0');
        else if (c >= 'a' && c <= 'f') v |= (uint32_t)(c - 'a' + 10);
        else if (c >= 'A' && c <= 'F') v |= (uint32_t)(c - 'A' + 10);
        else return -1;
    }
    ps->p += 4;
    *out = v;
    return 0;
}

static int parse_string(Parser* ps, char** out) {
    if (ps->p >= ps->end || *ps->p != '"') return fail(ps, "expected a string");
    ++ps->p;
    char* buf = NULL;
    size_t len = 0, cap = 0;
    if (put_utf8(&buf, &len, &cap, 0) != 0) return fail(ps, "out of memory");
    len = 0;
    while (ps->p < ps->end && *ps->p != '"') {
        uint32_t cp = (unsigned char)*ps->p++;
        if (cp < 0x20) { free(buf); return fail(ps, "control character in a string"); }
        if (cp == '\\') {
            if (ps->p >= ps->end) break;
            const char e = *ps->p++;
            switch (e) {
                case '"': cp = '"'; break;
                case '\\': cp = '\\'; break;
                case '/': cp = '/'; break;
                case 'b': cp = 8; break;
                case 'f': cp = 12; break;
                case 'n': cp = 10; break;
                case 'r': cp = 13; break;
                case 't': cp = 9; break;
                case 'u': {
                    if (hex4(ps, &cp) != 0) { free(buf); return fail(ps, "bad \\u escape"); }
                    if (cp >= 0xD800 && cp < 0xDC00) {   /* surrogate pair */
                        uint32_t lo = 0;
                        if (ps->end - ps->p < 6 || ps->p[0] != '\\' || ps->p[1] != 'u') {
                            free(buf);
                            return fail(ps, "unpaired surrogate");
                        }
                        ps->p += 2;
                        if (hex4(ps, &lo) != 0 || lo < 0xDC00 || lo >= 0xE000) {
                            free(buf);
                            return fail(ps, "bad surrogate pair");
                        }
                        cp = 0x10000 + ((cp - 0xD800) << 10) + (lo - 0xDC00);
                    }
                    break;
                }
                default: free(buf); return fail(ps, "bad escape");
            }
            if (put_utf8(&buf, &len, &cap, cp) != 0) { free(buf); return fail(ps, "out of memory"); }
        } else {
            /* raw byte (UTF-8 passes through unchanged) */
            if (len + 2 > cap) {
                char* nb = (char*)realloc(buf, cap * 2);
                if (!nb) { free(buf); return fail(ps, "out of memory"); }
                buf = nb;
                cap *= 2;
            }
            buf[len++] = (char)cp;
            buf[len] = '\0';
        }
    }
    if (ps->p >= ps->end) { free(buf); return fail(ps, "unterminated string"); }
    ++ps->p;
    *out = buf;
    return 0;
}

static int parse_value(Parser* ps, RoverJson* v);

static int push_item(RoverJson* v, int* cap) {
    if (v->count == *cap) {
        const int c = *cap ? *cap * 2 : 8;
        RoverJson* items = (RoverJson*)realloc(v->items, (size_t)c * sizeof(RoverJson));
        if (!items) return -1;
        v->items = items;
        if (v->kind == ROVER_JSON_OBJECT) {
            char** keys = (char**)realloc(v->keys, (size_t)c * sizeof(char*));
            if (!keys) return -1;
            v->keys = keys;
        }
        *cap = c;
    }
    memset(&v->items[v->count], 0, sizeof(RoverJson));
    if (v->kind == ROVER_JSON_OBJECT) v->keys[v->count] = NULL;
    ++v->count;
    return 0;
}

static int parse_value(Parser* ps, RoverJson* v) {
    memset(v, 0, sizeof(*v));
    if (++ps->depth > 64) return fail(ps, "nesting too deep");
    skip_ws(ps);
    if (ps->p >= ps->end) return fail(ps, "unexpected end");
    const char c = *ps->p;
    int rc = 0;
    if (c == '{' || c == '[') {
        const int object = c == '{';
        const char close = object ? '}' : ']';
        v->kind = object ? ROVER_JSON_OBJECT : ROVER_JSON_ARRAY;
        ++ps->p;
        int cap = 0;
        skip_ws(ps);
        if (ps->p < ps->end && *ps->p == close) {
            ++ps->p;
        } else {
            for (;;) {
                if (push_item(v, &cap) != 0) return fail(ps, "out of memory");
                skip_ws(ps);
                if (object) {
                    if (parse_string(ps, &v->keys[v->count - 1]) != 0) return -1;
                    skip_ws(ps);
                    if (ps->p >= ps->end || *ps->p != ':') return fail(ps, "expected ':'");
                    ++ps->p;
                }
                if (parse_value(ps, &v->items[v->count - 1]) != 0) return -1;
                skip_ws(ps);
                if (ps->p < ps->end && *ps->p == ',') { ++ps->p; continue; }
                if (ps->p < ps->end && *ps->p == close) { ++ps->p; break; }
                return fail(ps, object ? "expected ',' or '}'" : "expected ',' or ']'");
            }
        }
    } else if (c == '"') {
        v->kind = ROVER_JSON_STRING;
        rc = parse_string(ps, &v->str);
    } else if (c == 't' && ps->end - ps->p >= 4 && !memcmp(ps->p, "true", 4)) {
        v->kind = ROVER_JSON_BOOL; v->boolean = 1; ps->p += 4;
    } else if (c == 'f' && ps->end - ps->p >= 5 && !memcmp(ps->p, "false", 5)) {
        v->kind = ROVER_JSON_BOOL; v->boolean = 0; ps->p += 5;
    } else if (c == 'n' && ps->end - ps->p >= 4 && !memcmp(ps->p, "null", 4)) {
        v->kind = ROVER_JSON_NULL; ps->p += 4;
    } else if (c == '-' || (c >= '0' && c <= '9')) {
        /* the RFC grammar, then strtod on the validated span */
        const char* s = ps->p;
        const char* q = s;
        if (q < ps->end && *q == '-') ++q;
        if (q < ps->end && *q == '0') ++q;
        else if (q < ps->end && *q >= '1' && *q <= '9') while (q < ps->end && *q >= '0' && *q <= '9') ++q;
        else return fail(ps, "bad number");
        if (q < ps->end && *q == '.') {
            ++q;
            if (q >= ps->end || *q < '0' || *q > '9') return fail(ps, "bad number");
            while (q < ps->end && *q >= '0' && *q <= '9') ++q;
        }
        if (q < ps->end && (*q == 'e' || *q == 'E')) {
            ++q;
            if (q < ps->end && (*q == '+' || *q == '-')) ++q;
            if (q >= ps->end || *q < '0' || *q > '9') return fail(ps, "bad number");
            while (q < ps->end && *q >= '0' && *q <= '9') ++q;
        }
        char tmp[64];
        const size_t n = (size_t)(q - s);
        if (n >= sizeof(tmp)) return fail(ps, "number too long");
        memcpy(tmp, s, n);
        tmp[n] = '\0';
        v->kind = ROVER_JSON_NUMBER;
        v->num = strtod(tmp, NULL);
        ps->p = q;
    } else {
        return fail(ps, "unexpected character");
    }
    --ps->depth;
    return rc;
}

void rover_json_free(RoverJson* v) {
    if (!v) return;
    for (int i = 0; i < v->count; ++i) {
        rover_json_free(&v->items[i]);
        if (v->keys) free(v->keys[i]);
    }
    free(v->items);
    free(v->keys);
    free(v->str);
    memset(v, 0, sizeof(*v));
}

int rover_json_parse(const char* text, size_t len, RoverJson* out, char* err, size_t errlen) {
    Parser ps = {text, text + len, err, errlen, 0};
    if (parse_value(&ps, out) != 0) {
        rover_json_free(out);
        return -1;
    }
    skip_ws(&ps);
    if (ps.p != ps.end) {
        rover_json_free(out);
        return fail(&ps, "trailing characters");
    }
    return 0;
}

const RoverJson* rover_json_get(const RoverJson* obj, const char* key) {
    if (!obj || obj->kind != ROVER_JSON_OBJECT) return NULL;
    for (int i = 0; i < obj->count; ++i)
        if (obj->keys[i] && !strcmp(obj->keys[i], key)) return &obj->items[i];
    return NULL;
}
