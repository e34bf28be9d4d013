/* lua_host.c -- a minimal embedding of Lua 5.2 with the modules a Mara driver script uses,
 * in the way ctf-core/ctf.c:130-160 sets up its interpreter: `Mara` (this project's
 * lmara_gpu.c) and `buffer` (the reference's ctf-core/lua-buffer.c, unchanged) preloaded as
 * globals.  It is what the Lua drop-in is tested through; a maintainer instead links
 * lmara_gpu.o into the reference's ctf-main in place of Mara/mara.o.
 *
 * C API (for ctypes): mlua_open, mlua_dostring, mlua_error, mlua_close. */
#include <string.h>

#include "lua.h"
#include "lauxlib.h"
#include "lualib.h"

int luaopen_Mara(lua_State *L);
int luaopen_buffer(lua_State *L);

static char last_error[4096];

lua_State *mlua_open(void)
{
  lua_State *L = luaL_newstate();
  if (!L) return NULL;
  luaL_openlibs(L);
  luaL_requiref(L, "Mara", luaopen_Mara, 1);
  lua_pop(L, 1);
  luaL_requiref(L, "buffer", luaopen_buffer, 1);
  lua_pop(L, 1);
  return L;
}

int mlua_dostring(lua_State *L, const char *code)
{
  if (!L || !code) return 1;
  if (luaL_dostring(L, code)) {
    const char *m = lua_tostring(L, -1);
    strncpy(last_error, m ? m : "(no message)", sizeof(last_error) - 1);
    last_error[sizeof(last_error) - 1] = '\0';
    lua_pop(L, 1);
    return 1;
  }
  last_error[0] = '\0';
  return 0;
}

const char *mlua_error(void) { return last_error; }

void mlua_close(lua_State *L)
{
  if (L) lua_close(L);
}
