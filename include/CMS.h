/* The reference's main.c includes libCMS's umbrella header (main.c:7). The
 * engine parses basis sets, molecules and SAD guesses itself, so nothing of
 * libCMS is part of this API; the header exists so main.c compiles unchanged. */
#ifndef TINYSCF_B200_CMS_H
#define TINYSCF_B200_CMS_H
#endif
