/* Test infrastructure: opaque stand-ins for the three types of the lime
   library that the reference's ILDG headers (lib/IO/ILDG_reader.hpp,
   ILDG_writer.hpp) name through pointers.  Lime is not installed, so the ILDG
   reader and writer are not compiled; these declarations only let the headers
   that include them (lib/IO/readers.hpp, writers.hpp, fields_io.hpp) parse. */
#ifndef ORACLE_LIME_STANDIN_H
#define ORACLE_LIME_STANDIN_H
typedef struct LimeReader LimeReader;
typedef struct LimeWriter LimeWriter;
typedef struct LimeRecordHeader LimeRecordHeader;
#endif
