/* json.h -- the JSON reader of the bundle loader (internal to librover_host). */
#ifndef ROVER_HOST_JSON_H
#define ROVER_HOST_JSON_H

#include <stddef.h>
#include <stdint.h>

typedef enum {
    ROVER_JSON_NULL, ROVER_JSON_BOOL, ROVER_JSON_NUMBER, ROVER_JSON_STRING, ROVER_JSON_ARRAY, ROVER_JSON_OBJECT
} RoverJsonKind;

typedef struct RoverJson {
    RoverJsonKind kind;
    int boolean;
    double num;
    char *str;                 /* STRING: NUL-terminated UTF-8 */
    int count;                 /* ARRAY / OBJECT members */
    char **keys;               /* OBJECT keys */
    struct RoverJson *items;
} RoverJson;

int rover_json_parse(const char *text, size_t len, RoverJson *out, char *err, size_t errlen);
const RoverJson *rover_json_get(const RoverJson *obj, const char *key);
void rover_json_free(RoverJson *v);

#endif
