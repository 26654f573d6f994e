/* The reference includes <clapack.h> but calls no CLAPACK routine; an empty header satisfies the include. */
