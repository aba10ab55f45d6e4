/* Empty stand-in (the reference includes it but calls nothing from it).  TEST INFRASTRUCTURE ONLY. */
